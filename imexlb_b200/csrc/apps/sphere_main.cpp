// Sphere driver: the call sequence of sphere/main.cpp (System with
// Time = (2R)^2/miu and inter = 1, LBM, Initialize, the step loop; the
// reference's output calls are commented out, so output is off unless
// --inter is given).
#include "driver.h"

int main(int argc, char** argv) {
  driver::Options o = driver::parse(argc, argv);
  imexlb_system s;
  driver::check(imexlb_system_read("input.in", IMEXLB_SPHERE, &s), "reading input.in");
  driver::monitor(s);
  const int steps = o.steps > 0 ? o.steps : s.Time;
  imexlb_lattice* h = driver::make(IMEXLB_SPHERE, s, o);
  const auto t0 = std::chrono::steady_clock::now();
  if (o.inter > 0) {
    for (int it = 1; it <= steps;) {
      const int n = std::min(o.inter, steps - it + 1);
      driver::check(imexlb_step(h, n), "step");
      it += n;
      if (o.output) {
        const std::string name = "output" + std::to_string((it - 1) / o.inter) + ".plt";
        driver::check(imexlb_write_tecplot(h, name.c_str(), (it - 1) / o.inter), "MPIoutput");
      }
    }
  } else {
    driver::check(imexlb_step(h, steps), "step");
  }
  driver::check(imexlb_synchronize(h), "step");
  const double total = driver::seconds_since(t0);
  std::printf("MLUPS: %.1f\n", static_cast<double>(s.sx) * s.sy * s.sz * steps / total / 1e6);
  imexlb_destroy(h);
  return 0;
}
