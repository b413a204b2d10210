// Shared pieces of the three case drivers (tgv, cavity, sphere), which keep
// the reference proxy apps' driver surface: they read input.in from the
// working directory, print System's monitor banner, and run the reference's
// call sequence through the C ABI of include/imexlb.h.
//
// Options (all optional; without them the drivers behave like the
// reference's main() at one rank):
//   --steps N        override the step count (System's Time)
//   --inter N        output interval (System's inter)
//   --storage f64|f32|f16|bf16
//   --bc reference|reference-links|standard
//   --arith exact|fast
//   --no-output      do not write output<n>.plt
#pragma once

#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <algorithm>
#include <string>

#include "imexlb.h"

namespace driver {

struct Options {
  int steps = -1;
  int inter = -1;
  imexlb_storage storage = IMEXLB_F64;
  imexlb_bc bc = IMEXLB_BC_REFERENCE;
  imexlb_arith arith = IMEXLB_ARITH_EXACT;
  bool output = true;
};

inline Options parse(int argc, char** argv) {
  Options o;
  for (int a = 1; a < argc; ++a) {
    const std::string s = argv[a];
    auto next = [&]() -> std::string {
      if (a + 1 >= argc) {
        std::fprintf(stderr, "missing value after %s\n", s.c_str());
        std::exit(2);
      }
      return argv[++a];
    };
    if (s == "--steps") o.steps = std::atoi(next().c_str());
    else if (s == "--inter") o.inter = std::atoi(next().c_str());
    else if (s == "--no-output") o.output = false;
    else if (s == "--storage") {
      const std::string v = next();
      o.storage = v == "f32" ? IMEXLB_F32 : v == "f16" ? IMEXLB_F16 : v == "bf16" ? IMEXLB_BF16 : IMEXLB_F64;
    } else if (s == "--bc") {
      const std::string v = next();
      o.bc = v == "standard" ? IMEXLB_BC_STANDARD : v == "reference-links" ? IMEXLB_BC_REFERENCE_LINKS
                                                                             : IMEXLB_BC_REFERENCE;
    } else if (s == "--arith") {
      o.arith = next() == "fast" ? IMEXLB_ARITH_FAST : IMEXLB_ARITH_EXACT;
    } else {
      std::fprintf(stderr, "unknown option %s\n", s.c_str());
      std::exit(2);
    }
  }
  return o;
}

inline void check(int rc, const char* what) {
  if (rc != IMEXLB_OK) {
    std::fprintf(stderr, "%s failed (%d): %s\n", what, rc, imexlb_last_error());
    std::exit(1);
  }
}

// System::Monitor (tgv/src/System.cpp:26-42), banner text kept as printed
inline void monitor(const imexlb_system& s) {
  std::printf("============================\n3D Cylinder Flow\nRe    =%d\nMa    =%g\nrho   =%g\nmiu   =%g\n"
              "tau   =%g\nTime  =%d\ninter =%d\nnx    =%d\nny    =%d\nnz    =%d\n============================\n",
              s.Re, s.Ma, s.rho0, s.miu, s.tau, s.Time, s.inter, s.sx, s.sy, s.sz);
}

inline imexlb_lattice* make(imexlb_case kase, const imexlb_system& s, const Options& o) {
  imexlb_params p;
  imexlb_params_default(&p);
  p.kase = kase;
  p.bc = o.bc;
  p.storage = o.storage;
  p.arith = o.arith;
  p.nx = s.sx;
  p.ny = s.sy;
  p.nz = s.sz;
  p.tau0 = s.tau;
  p.rho0 = s.rho0;
  p.u0 = s.u0;
  imexlb_lattice* h = nullptr;
  check(imexlb_create(&p, &h), "imexlb_create");
  return h;
}

inline double seconds_since(std::chrono::steady_clock::time_point t0) {
  return std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
}

}  // namespace driver
