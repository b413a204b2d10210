// Taylor-Green vortex driver: the call sequence of tgv/main.cpp:37-206 at one
// rank -- System, LBM, Initialize, 20 warm-up steps, Initialize again, the
// timed loop (Time = 100 unless --steps), then the average time per step.
#include "driver.h"

int main(int argc, char** argv) {
  const driver::Options o = driver::parse(argc, argv);
  imexlb_system s;
  driver::check(imexlb_system_read("input.in", IMEXLB_TGV, &s), "reading input.in");
  std::printf("System Definition: Done\n");
  driver::monitor(s);
  const int steps = o.steps > 0 ? o.steps : s.Time;
  imexlb_lattice* h = driver::make(IMEXLB_TGV, s, o);
  std::printf("Warm-Up\n");
  driver::check(imexlb_step(h, 20), "warm-up");
  driver::check(imexlb_synchronize(h), "warm-up");
  std::printf("Reset and Run Main-Loop\n");
  driver::check(imexlb_initialize(h), "Initialize");
  const auto t0 = std::chrono::steady_clock::now();
  driver::check(imexlb_step(h, steps), "step");
  driver::check(imexlb_synchronize(h), "step");
  const double total = driver::seconds_since(t0);
  const double cells = static_cast<double>(s.sx) * s.sy * s.sz;
  std::printf("Avg. Total Solver Time:  %lf\n", total);
  std::printf("Avg. Time per time-step:  %lf\n", total / steps);
  std::printf("MLUPS: %.1f\n", cells * steps / total / 1e6);
  if (o.output && o.inter > 0) driver::check(imexlb_write_tecplot(h, "output1.plt", 1), "MPIoutput");
  imexlb_destroy(h);
  return 0;
}
