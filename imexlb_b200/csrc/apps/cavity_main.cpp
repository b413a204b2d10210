// Lid-driven cavity driver: the call sequence of lid_driven_cavity/main.cpp:
// System, LBM, Initialize, MPIoutput(0), then Time steps with MPIoutput(it /
// inter) every `inter` steps and the elapsed time printed with each output.
#include "driver.h"

int main(int argc, char** argv) {
  const driver::Options o = driver::parse(argc, argv);
  imexlb_system s;
  driver::check(imexlb_system_read("input.in", IMEXLB_CAVITY, &s), "reading input.in");
  driver::monitor(s);
  const int steps = o.steps > 0 ? o.steps : s.Time;
  const int inter = o.inter > 0 ? o.inter : s.inter;
  imexlb_lattice* h = driver::make(IMEXLB_CAVITY, s, o);
  if (o.output) driver::check(imexlb_write_tecplot(h, "output0.plt", 0), "MPIoutput");
  const auto t0 = std::chrono::steady_clock::now();
  for (int it = 1; it <= steps;) {
    const int n = std::min(inter - (it - 1) % inter, steps - it + 1);
    driver::check(imexlb_step(h, n), "step");
    it += n;
    if ((it - 1) % inter == 0) {
      driver::check(imexlb_synchronize(h), "step");
      if (o.output) {
        const std::string name = "output" + std::to_string((it - 1) / inter) + ".plt";
        driver::check(imexlb_write_tecplot(h, name.c_str(), (it - 1) / inter), "MPIoutput");
      }
      std::printf("time=%f\n", driver::seconds_since(t0));
    }
  }
  driver::check(imexlb_synchronize(h), "step");
  const double total = driver::seconds_since(t0);
  std::printf("MLUPS: %.1f\n", static_cast<double>(s.sx) * s.sy * s.sz * steps / total / 1e6);
  imexlb_destroy(h);
  return 0;
}
