// The multimethod layer alone (no GPU): registration, most-specific
// resolution over two virtual arguments, fallback overloads, methods that
// share a name with different signatures, ambiguity reported as
// frank_mm::dispatch_error.  Exit status 0 only if every check passes.
#include "frank_b200/multimethod.hpp"

#include <cstdio>
#include <string>

using frank_mm::virtual_;

struct Shape { virtual ~Shape() = default; };
struct Box : Shape {};
struct Cube : Box {};
struct Ball : Shape {};

register_class(Shape)
register_class(Box, Shape)
register_class(Cube, Box)
register_class(Ball, Shape)

declare_method(std::string, meet, (virtual_<const Shape&>, virtual_<const Shape&>))
define_method(std::string, meet, (const Shape&, const Shape&)) { return "shape-shape"; }
define_method(std::string, meet, (const Box&, const Shape&)) { return "box-shape"; }
define_method(std::string, meet, (const Box&, const Box&)) { return "box-box"; }
define_method(std::string, meet, (const Cube&, const Ball&)) { return "cube-ball"; }
define_method(std::string, meet, (const Shape&, const Ball&)) { return "shape-ball"; }

// same name, another signature (FRANK's two gemm_omm)
declare_method(int, meet, (virtual_<Shape&>, int))
define_method(int, meet, (Box&, int k)) { return 10 + k; }
define_method(int, meet, (Shape&, int k)) { return k; }

static int failures = 0;
static void expect(bool ok, const char* what) {
  std::printf("%s %s\n", ok ? "PASS" : "FAIL", what);
  if (!ok) ++failures;
}

int main() {
  Shape s;
  Box b;
  Cube c;
  Ball l;
  const Shape& rs = s; const Shape& rb = b; const Shape& rc = c; const Shape& rl = l;
  expect(meet(rs, rs) == "shape-shape", "fallback");
  expect(meet(rb, rs) == "box-shape", "first argument more specific");
  expect(meet(rc, rb) == "box-box", "inherited overload through a registered base");
  expect(meet(rc, rl) == "cube-ball", "most specific in both arguments");
  expect(meet(rs, rl) == "shape-ball", "second argument more specific");
  bool amb = false;
  try {
    meet(rb, rl);   // (Box, Shape) vs (Shape, Ball): neither is more specific
  } catch (const frank_mm::dispatch_error& e) {
    amb = std::string(e.what()).find("ambiguous") != std::string::npos;
  }
  expect(amb, "ambiguity is an error");
  Shape& ws = s; Shape& wc = c;
  expect(meet(wc, 5) == 15 && meet(ws, 5) == 5, "overloaded method name, second signature");
  std::printf("%d failures\n", failures);
  return failures == 0 ? 0 : 1;
}
