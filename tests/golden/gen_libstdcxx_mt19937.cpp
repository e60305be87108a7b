// Prints std::mt19937 / libstdc++ distribution outputs used as golden vectors.
#include <random>
#include <cstdio>
int main(){
  { std::mt19937 g; g.seed(0); for(int i=0;i<8;i++) printf("raw %u\n",(unsigned)g()); }
  { std::mt19937 g; g.seed(0); std::uniform_real_distribution<> d(0,1); for(int i=0;i<16;i++) printf("uniform %.17g\n", d(g)); }
  { std::mt19937 g; g.seed(0); std::normal_distribution<double> d(0.0,1.0); for(int i=0;i<16;i++) printf("normal %.17g\n", d(g)); }
}
