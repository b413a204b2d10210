// Stand-in for Kokkos::Random_XorShift64_Pool (Kokkos 4.0.01, not present
// here).  Only sphere/src/lbm.cpp:221-228 uses it, to fill the integer field
// `ran` with urand(100).  Kokkos' own pool hands out per-thread states whose
// assignment to cells depends on scheduling, so no CPU run can reproduce the
// values of a given GPU run; this project therefore treats `ran` as an input
// field.  The stand-in is a single shared xorshift64* stream (Vigna, "An
// experimental exploration of Marsaglia's xorshift generators", 2016), which
// makes the reference run here deterministic when it runs on one thread.
#pragma once
#include <cstdint>
#include <memory>
#include <mutex>

namespace Kokkos {

template <class Device = void>
class Random_XorShift64_Pool {
 public:
  class generator_type {
   public:
    uint64_t s = 1;
    uint64_t next() {
      s ^= s >> 12;
      s ^= s << 25;
      s ^= s >> 27;
      return s * 2685821657736338717ULL;
    }
    uint32_t urand() { return static_cast<uint32_t>(next() >> 32); }
    uint32_t urand(uint32_t range) { return urand() % range; }
    double drand() { return (next() >> 11) * (1.0 / 9007199254740992.0); }
  };

  explicit Random_XorShift64_Pool(uint64_t seed)
      : st_(std::make_shared<State>()) {
    st_->g.s = seed ? seed : 1318319ULL;
  }
  generator_type get_state() const {
    st_->m.lock();
    return st_->g;
  }
  void free_state(const generator_type& g) const {
    st_->g = g;
    st_->m.unlock();
  }

 private:
  struct State {
    generator_type g;
    std::mutex m;
  };
  std::shared_ptr<State> st_;
};

template <class G, class S> struct rand {
  static S draw(G& g) { return static_cast<S>(g.drand()); }
};

}  // namespace Kokkos
