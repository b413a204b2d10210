// Ghost-slot plan of the reference boundary passes.
//
// At one rank the reference fills ghost slots every step with a fixed
// sequence of copy passes between Collision and the pull:
//   cavity  unpack of four never-received planes (zeroed),
//           bcl, bcr, bcf, bcb, bcd, bcu   (lid_driven_cavity/src/mpi_view_transfer.cpp:598-690,
//                                           lid_driven_cavity/src/lbm.cpp:231-301)
//   sphere  bcf, bcb, bcd, bcu, bcl, bcr, usrbc      (sphere/src/lbm.cpp:274-356)
// Each pass copies a slot f(q', x') into a slot f(q, x).  Because later passes
// read slots written by earlier ones (and by earlier steps), a slot's value is
// a chain of copies ending at a post-collision interior slot of this step, a
// ghost slot as it stood before this step's passes, or zero.  This file runs
// the pass sequence once on provenance tags instead of values and keeps, for
// every ghost slot the next pull (or a later step's chain) can reach, where
// its value comes from.  The device then applies the whole sequence as one
// gather per step (kernels.cu, ghost_gather_kernel).
#include <string>
#include <unordered_map>
#include <unordered_set>
#include <vector>

#include "lattice.h"

namespace imx {
namespace {

constexpr int64_t ZERO_TAG = -1;

struct Tracer {
  int kase, nx, ny, nz, lx, ly, lz;
  const int32_t* usr;  // padded mask or null
  std::unordered_map<int64_t, int64_t> tag;  // slots written this step -> source tag

  int64_t key(int q, int i, int j, int k) const {
    return q + static_cast<int64_t>(Q) * (i + static_cast<int64_t>(lx) * (j + static_cast<int64_t>(ly) * k));
  }
  bool interior(int i, int j, int k) const {
    return i >= GHOST && i < GHOST + nx && j >= GHOST && j < GHOST + ny && k >= GHOST && k < GHOST + nz;
  }
  // The cavity's unpack writes zero into planes y = l_e1, z = l_e2, x = l_s0-1
  // and x = l_e0 before any boundary pass (one rank).
  bool zero_plane(int i, int j, int k) const {
    return kase == 1 && (j == GHOST + ny || k == GHOST + nz || i == GHOST - 1 || i == GHOST + nx);
  }
  // Tag of a slot at the start of the pass sequence.
  int64_t initial(int q, int i, int j, int k) const {
    const int64_t kk = key(q, i, j, k);
    if (interior(i, j, k)) return kk;  // this step's post-collision value
    if (zero_plane(i, j, k)) return ZERO_TAG;
    return -kk - 2;  // value before this step
  }
  int64_t get(int q, int i, int j, int k) const {
    auto it = tag.find(key(q, i, j, k));
    return it != tag.end() ? it->second : initial(q, i, j, k);
  }
  bool in_box(int i, int j, int k) const { return i >= 0 && i < lx && j >= 0 && j < ly && k >= 0 && k < lz; }
};

struct Pass {
  std::vector<std::pair<int64_t, int64_t>> w;  // (target key, source tag)
  std::unordered_set<int64_t> targets;
  std::vector<int64_t> sources;  // source keys read by this pass
};

// A pass reads everything before it writes (the parallel kernel's
// semantics); if it reads a slot it also writes, its outcome would depend on
// thread order and the plan is refused.
bool apply(Tracer& t, Pass& p, const char* name, std::string* err) {
  for (int64_t s : p.sources)
    if (p.targets.count(s)) {
      *err = std::string("boundary pass ") + name + " reads a slot it writes (order-dependent result)";
      return false;
    }
  for (auto& e : p.w) t.tag[e.first] = e.second;
  return true;
}

void copy_into(Tracer& t, Pass& p, int q, int i, int j, int k, int qs, int is, int js, int ks) {
  const int64_t tk = t.key(q, i, j, k);
  p.w.emplace_back(tk, t.get(qs, is, js, ks));
  p.targets.insert(tk);
  p.sources.push_back(t.key(qs, is, js, ks));
}

// Mirror passes: ghost layer g (one below the interior on the low side,
// one above on the high side) over the tangential range [2, L-2), source
// f(bb(q), g + 2 e_q) with the tangential y step scaled by `jscale_y` (the
// cavity's top wall uses j + e_y; lid_driven_cavity/src/lbm.cpp:298).
bool wall_pass(Tracer& t, int axis, bool low, int jscale_y, const char* name, std::string* err) {
  Pass p;
  const int n[3] = {t.nx, t.ny, t.nz};
  const int L[3] = {t.lx, t.ly, t.lz};
  const int g = low ? GHOST - 1 : GHOST + n[axis];
  const int src_n = low ? GHOST + 1 : GHOST + n[axis] - 2;
  const int sign = low ? 1 : -1;
  const int a1 = axis == 0 ? 1 : 0, a2 = axis == 2 ? 1 : 2;
  for (int q = 0; q < Q; ++q) {
    const int e[3] = {D3Q27::ex[q], D3Q27::ey[q], D3Q27::ez[q]};
    if (e[axis] * sign <= 0) continue;
    for (int c2 = GHOST - 1; c2 < L[a2] - GHOST + 1; ++c2)
      for (int c1 = GHOST - 1; c1 < L[a1] - GHOST + 1; ++c1) {
        int x[3], s[3];
        x[axis] = g;
        x[a1] = c1;
        x[a2] = c2;
        s[axis] = src_n;
        s[a1] = c1 + (a1 == 1 ? jscale_y : 2) * e[a1];
        s[a2] = c2 + (a2 == 1 ? jscale_y : 2) * e[a2];
        copy_into(t, p, q, x[0], x[1], x[2], D3Q27::bb[q], s[0], s[1], s[2]);
      }
  }
  return apply(t, p, name, err);
}

}  // namespace

bool build_ghost_plan_keys(int kase, int nx, int ny, int nz, const int32_t* usr_padded, GhostPlan* out,
                           std::string* err) {
  Tracer t{kase, nx, ny, nz, nx + 2 * GHOST, ny + 2 * GHOST, nz + 2 * GHOST, usr_padded, {}};
  out->tgt.clear();
  out->src.clear();
  if (kase == 1) {
    if (!wall_pass(t, 0, true, 2, "bcl", err) || !wall_pass(t, 0, false, 2, "bcr", err) ||
        !wall_pass(t, 1, true, 2, "bcf", err) || !wall_pass(t, 1, false, 2, "bcb", err) ||
        !wall_pass(t, 2, true, 2, "bcd", err) || !wall_pass(t, 2, false, 1, "bcu", err))
      return false;
  } else if (kase == 2) {
    if (!wall_pass(t, 1, true, 2, "bcf", err) || !wall_pass(t, 1, false, 2, "bcb", err) ||
        !wall_pass(t, 2, true, 2, "bcd", err) || !wall_pass(t, 2, false, 2, "bcu", err))
      return false;
    {  // bcl: inlet ghost plane copies the first interior plane (sphere/src/lbm.cpp:326-335)
      Pass p;
      for (int q = 0; q < Q; ++q) {
        if (D3Q27::ex[q] <= 0) continue;
        for (int k = GHOST - 1; k < t.lz - GHOST + 1; ++k)
          for (int j = GHOST - 1; j < t.ly - GHOST + 1; ++j) copy_into(t, p, q, GHOST - 1, j, k, q, GHOST, j, k);
      }
      if (!apply(t, p, "bcl", err)) return false;
    }
    {  // bcr: outlet ghost plane takes f(q, x + e) (sphere/src/lbm.cpp:338-347)
      Pass p;
      const int xe = GHOST + nx;
      for (int q = 0; q < Q; ++q) {
        if (D3Q27::ex[q] >= 0) continue;
        for (int k = GHOST - 1; k < t.lz - GHOST + 1; ++k)
          for (int j = GHOST - 1; j < t.ly - GHOST + 1; ++j)
            copy_into(t, p, q, xe, j, k, q, xe + D3Q27::ex[q], j + D3Q27::ey[q], k + D3Q27::ez[q]);
      }
      if (!apply(t, p, "bcr", err)) return false;
    }
    if (usr_padded) {  // usrbc (sphere/src/lbm.cpp:350-356)
      Pass p;
      auto U = [&](int i, int j, int k) {
        return usr_padded[i + static_cast<int64_t>(t.lx) * (j + static_cast<int64_t>(t.ly) * k)];
      };
      for (int k = GHOST; k < t.lz - GHOST; ++k)
        for (int j = GHOST; j < t.ly - GHOST; ++j)
          for (int i = GHOST; i < t.lx - GHOST; ++i) {
            if (U(i, j, k) != 0) continue;
            for (int q = 0; q < Q; ++q) {
              const int a = i + D3Q27::ex[q], b = j + D3Q27::ey[q], c = k + D3Q27::ez[q];
              if (U(a, b, c) != 1) continue;
              copy_into(t, p, q, i, j, k, D3Q27::bb[q], i + 2 * D3Q27::ex[q], j + 2 * D3Q27::ey[q],
                        k + 2 * D3Q27::ez[q]);
            }
          }
      if (!apply(t, p, "usrbc", err)) return false;
    }
  } else {
    return true;  // periodic case: no ghost slots
  }

  // Slots whose value must be materialised after a step: every rewritten slot
  // an interior cell pulls (ghost slots of the one-cell shell and the
  // sphere's solid cells), then, transitively, every slot written each step
  // whose previous value such a slot is copied from.
  auto final_tag = [&](int64_t k, int q, int i, int j, int kk) {
    auto it = t.tag.find(k);
    return it != t.tag.end() ? it->second : t.initial(q, i, j, kk);
  };
  auto decode_key = [&](int64_t k, int& q, int& i, int& j, int& kk) {
    q = static_cast<int>(k % Q);
    int64_t c = k / Q;
    i = static_cast<int>(c % t.lx);
    c /= t.lx;
    j = static_cast<int>(c % t.ly);
    kk = static_cast<int>(c / t.ly);
  };
  auto written = [&](int64_t k, int i, int j, int kk) { return t.tag.count(k) || t.zero_plane(i, j, kk); };

  std::unordered_set<int64_t> emitted;
  std::vector<int64_t> work;
  auto emit = [&](int64_t k) {
    if (!emitted.insert(k).second) return;
    int q, i, j, kk;
    decode_key(k, q, i, j, kk);
    const int64_t src = final_tag(k, q, i, j, kk);
    out->tgt.push_back(k);
    out->src.push_back(src);
    if (src <= -2) work.push_back(-src - 2);
  };
  for (int k = GHOST - 1; k <= GHOST + nz; ++k)
    for (int j = GHOST - 1; j <= GHOST + ny; ++j)
      for (int i = GHOST - 1; i <= GHOST + nx; ++i) {
        if (t.interior(i, j, k)) continue;
        for (int q = 0; q < Q; ++q) {
          if (!t.interior(i + D3Q27::ex[q], j + D3Q27::ey[q], k + D3Q27::ez[q])) continue;
          const int64_t kk = t.key(q, i, j, k);
          if (written(kk, i, j, k)) emit(kk);
        }
      }
  // interior slots rewritten by a pass (the sphere's solid cells, usrbc)
  for (const auto& kv : t.tag) {
    int q, i, j, kk;
    decode_key(kv.first, q, i, j, kk);
    if (t.interior(i, j, kk) && t.interior(i + D3Q27::ex[q], j + D3Q27::ey[q], kk + D3Q27::ez[q])) emit(kv.first);
  }
  while (!work.empty()) {
    const int64_t k = work.back();
    work.pop_back();
    int q, i, j, kk;
    decode_key(k, q, i, j, kk);
    if (written(k, i, j, kk)) emit(k);
  }
  // The gather reads this step's values at its interior sources while it
  // writes its targets; the two sets must not meet.
  for (int64_t s : out->src)
    if (s >= 0 && emitted.count(s)) {
      *err = "ghost plan: a copy source is also a copy target";
      return false;
    }
  return true;
}

}  // namespace imx
