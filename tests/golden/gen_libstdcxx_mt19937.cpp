// Prints std::mt19937 / std::mt19937_64 and libstdc++ distribution outputs
// used as golden vectors.
#include <random>
#include <cstdio>
int main(){
  { std::mt19937 g; g.seed(0); for(int i=0;i<8;i++) printf("raw %u\n",(unsigned)g()); }
  { std::mt19937 g; g.seed(0); std::uniform_real_distribution<> d(0,1); for(int i=0;i<16;i++) printf("uniform %.17g\n", d(g)); }
  { std::mt19937 g; g.seed(0); std::normal_distribution<double> d(0.0,1.0); for(int i=0;i<16;i++) printf("normal %.17g\n", d(g)); }
  { std::mt19937_64 g; g.seed(2); for(int i=0;i<700;i++) printf("raw64 %llu\n",(unsigned long long)g()); }
  { std::mt19937_64 g; g.seed(2); std::uniform_real_distribution<> d(0,1); for(int i=0;i<700;i++) printf("uniform64 %.17g\n", d(g)); }
  { std::mt19937_64 g; g.seed(3); std::normal_distribution<double> d(0.0,1.0); for(int i=0;i<700;i++) printf("normal64 %.17g\n", d(g)); }
}
