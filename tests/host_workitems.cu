// Host-side check of the engine's work lists (no GPU needed): the one-sweep
// work items of build_step_items and the deferred ADE pass's run list of
// build_ade_runs, on seeded random scenes.  Prints "ok <items> <runs>" and
// exits 0, or prints the first failures and exits 1.
#include <cstdio>
#include <random>
#include <vector>

#include "xfdtd_cuda_b200/csrc/engine.cuh"

using namespace xfb;

namespace {

int slab_of(int q, int n, int lo, int hi) { return q < lo ? q : (q >= n - hi ? lo + q - (n - hi) : -1); }

// region bits a kind index handles (1 x-slab, 2 y-slab, 8 z-slab, 4 ADE, 16 TFSF)
int kind_bits(int q) {
  if (q < 16) return kStepKinds[q];
  if (q == kFastY) return 3;
  if (q == kFastZ) return 9;
  if (q == kFastYZ) return 11;
  if (q == kFastYTf) return 3 | 16;
  if (q == kFastZTf) return 9 | 16;
  return 11 | 16;  // kFastYZTf
}

int bad = 0;
void fail(const char* what, int a, int b, int c, int d) {
  if (++bad <= 8) std::printf("FAIL %s (%d %d %d %d)\n", what, a, b, c, d);
}

Compiled random_scene(std::mt19937& rng, int trial) {
  Compiled c;
  c.dim = 3;
  if (trial == 0) {  // the 408^3 dispersive-sphere workload's layout
    c.nx = c.ny = c.nz = 408;
    for (int f = 0; f < 6; ++f) c.pml[f] = 12;
    c.ade_kind = XFB_ADE_MLORENTZ;
    const int bb[6] = {104, 304, 104, 304, 104, 304}, tt[6] = {27, 381, 27, 381, 27, 381};
    for (int q = 0; q < 6; ++q) { c.ade_box[q] = bb[q]; c.tf[q] = tt[q]; }
    c.tfsf_on = 1;
    return c;
  }
  c.nx = 8 + rng() % 90;
  c.ny = 8 + rng() % 90;
  c.nz = 8 + rng() % 130;
  for (int f = 0; f < 6; ++f) c.pml[f] = rng() % 3 ? rng() % 6 : 0;
  c.ade_kind = rng() % 2 ? XFB_ADE_DRUDE : XFB_ADE_NONE;
  const int n[3] = {c.nx, c.ny, c.nz};
  for (int a = 0; a < 3; ++a) {
    const int lo = rng() % n[a], hi = lo + rng() % (n[a] - lo + 1);
    c.ade_box[2 * a] = lo;
    c.ade_box[2 * a + 1] = hi;
    const int tlo = 1 + rng() % (n[a] - 2), thi = tlo + rng() % (n[a] - tlo);
    c.tf[2 * a] = tlo;
    c.tf[2 * a + 1] = thi;
  }
  c.tfsf_on = rng() % 3 != 0;
  return c;
}

long long check_items(const Compiled& c, int t, bool deferred, int trial) {
  const int TJ = kStepTiles[t].r * kStepTiles[t].nwm, NT = (kStepTiles[t].nwm + 1) * 32;
  std::vector<int4> items[kStepKindCount];
  build_step_items(c, TJ, NT, deferred, items, 0, true);
  const int gx = (c.nz + 31) / 32, gy = (c.ny + TJ - 1) / TJ;
  std::vector<int> cover(static_cast<size_t>(gx) * gy * c.nx, 0);
  const int* b = c.ade_box;
  const int* tt = c.tf;
  const bool ade_on = !deferred && c.ade_kind != XFB_ADE_NONE && b[1] > b[0];
  long long n = 0;
  for (int q = 0; q < kStepKindCount; ++q) {
    const int K = kind_bits(q);
    for (const int4& it : items[q]) {
      ++n;
      if (it.z >= it.w || it.z < 0 || it.w > c.nx || it.x >= gx || it.y >= gy) { fail("item range", trial, t, q, it.z); continue; }
      for (int p = it.z; p < it.w; ++p) cover[(static_cast<size_t>(it.y) * gx + it.x) * c.nx + p]++;
      const int j0 = it.y * TJ, k0 = it.x * 32;
      if ((q == kLeanInterior || q == kLeanInteriorTf) &&
          !(it.z >= 1 && j0 >= 1 && k0 >= 1 && j0 + TJ <= c.ny && k0 + 32 <= c.nz))
        fail("lean interior item not inside the grid", trial, t, j0, k0);
      // every cell the item updates (H from plane z-1, E from plane z; the
      // tile's halo row and column) needs no more than the kind handles
      for (int i = std::max(it.z - 1, 0); i < it.w; ++i)
        for (int j = std::max(j0 - 1, 0); j < std::min(j0 + TJ, c.ny); ++j)
          for (int k = std::max(k0 - 1, 0); k < std::min(k0 + 32, c.nz); ++k) {
            const bool px = slab_of(i, c.nx, c.pml[0], c.pml[1]) >= 0;
            const bool py = slab_of(j, c.ny, c.pml[2], c.pml[3]) >= 0;
            const bool pz = slab_of(k, c.nz, c.pml[4], c.pml[5]) >= 0;
            const bool e_cell = i >= it.z && j >= j0 && k >= k0;
            const bool ad = e_cell && ade_on && i >= b[0] && i < b[1] && j >= b[2] && j < b[3] && k >= b[4] && k < b[5];
            const bool iin = i >= tt[0] && i <= tt[1], jin = j >= tt[2] && j <= tt[3], kin = k >= tt[4] && k <= tt[5];
            const bool th = c.tfsf_on && (((i == tt[0] - 1 || i == tt[1]) && jin && kin) ||
                                          ((j == tt[2] - 1 || j == tt[3]) && iin && kin) ||
                                          ((k == tt[4] - 1 || k == tt[5]) && iin && jin));
            const bool te = c.tfsf_on && e_cell && (((i == tt[0] || i == tt[1]) && jin && kin) ||
                                                    ((j == tt[2] || j == tt[3]) && iin && kin) ||
                                                    ((k == tt[4] || k == tt[5]) && iin && jin));
            if ((th || te) && !(K & 16)) fail("kind without TFSF code meets a TFSF cell", trial, i, j, k);
            if ((px && !(K & 1)) || (py && !(K & 2)) || (pz && !(K & 8)) || (ad && !(K & 4)))
              fail("kind misses a CPML or ADE cell", trial, i, j, k);
          }
    }
  }
  for (size_t q = 0; q < cover.size(); ++q)
    if (cover[q] != 1) {
      fail("tile plane not covered exactly once", trial, t, static_cast<int>(q), cover[q]);
      break;
    }
  return n;
}

long long check_runs(std::mt19937& rng, int trial) {
  Compiled c;
  c.dim = 3;
  c.nx = 4 + rng() % 40;
  c.ny = 4 + rng() % 40;
  c.nz = 4 + rng() % 150;
  c.n_mat = 3;
  c.mat_disp = {0, 1, 1};
  c.mat_id.assign(static_cast<size_t>(c.nx) * c.ny * c.nz, 0);
  // a few random balls of dispersive material
  for (int s = 0; s < 3; ++s) {
    const double cx = rng() % c.nx, cy = rng() % c.ny, cz = rng() % c.nz, r = 2 + rng() % 20;
    const uint8_t m = static_cast<uint8_t>(1 + rng() % 2);
    for (int i = 0; i < c.nx; ++i)
      for (int j = 0; j < c.ny; ++j)
        for (int k = 0; k < c.nz; ++k)
          if ((i - cx) * (i - cx) + (j - cy) * (j - cy) + (k - cz) * (k - cz) <= r * r)
            c.mat_id[(static_cast<size_t>(i) * c.ny + j) * c.nz + k] = m;
  }
  // the box: bounds of the dispersive cells, widened at random
  int lo[3] = {c.nx, c.ny, c.nz}, hi[3] = {0, 0, 0};
  for (int i = 0; i < c.nx; ++i)
    for (int j = 0; j < c.ny; ++j)
      for (int k = 0; k < c.nz; ++k)
        if (c.mat_disp[c.mat_id[(static_cast<size_t>(i) * c.ny + j) * c.nz + k]]) {
          const int v[3] = {i, j, k};
          for (int a = 0; a < 3; ++a) { lo[a] = std::min(lo[a], v[a]); hi[a] = std::max(hi[a], v[a] + 1); }
        }
  const int n[3] = {c.nx, c.ny, c.nz};
  for (int a = 0; a < 3; ++a) {
    if (lo[a] >= hi[a]) { lo[a] = 0; hi[a] = 0; }
    c.ade_box[2 * a] = std::max(0, lo[a] - static_cast<int>(rng() % 3));
    c.ade_box[2 * a + 1] = std::min(n[a], hi[a] + static_cast<int>(rng() % 3));
  }
  std::vector<int2> runs;
  if (!build_ade_runs(c, runs)) { fail("no run list", trial, c.nx, c.ny, c.nz); return 0; }
  std::vector<int> seen(c.mat_id.size(), 0);
  long long prev = -1;
  for (const int2& r : runs) {
    const int i = r.x & 0xffff, j = static_cast<int>(static_cast<unsigned>(r.x) >> 16);
    const int kb = r.y & 0xffff, l0 = (r.y >> 16) & 0xff, l1 = static_cast<int>(static_cast<unsigned>(r.y) >> 24);
    if (kb % 32 != 0 || l0 >= l1 || l1 > 32 || i >= c.nx || j >= c.ny || kb + l1 > c.nz) {
      fail("run out of shape", trial, i, j, kb);
      continue;
    }
    const long long key = (static_cast<long long>(i) * c.ny + j) * c.nz + kb + l0;
    if (key <= prev) fail("runs out of (i, j, k) order", trial, i, j, kb + l0);
    prev = key;
    for (int k = kb + l0; k < kb + l1; ++k) seen[(static_cast<size_t>(i) * c.ny + j) * c.nz + k]++;
  }
  const int* b = c.ade_box;
  for (int i = 0; i < c.nx; ++i)
    for (int j = 0; j < c.ny; ++j)
      for (int k = 0; k < c.nz; ++k) {
        const size_t q = (static_cast<size_t>(i) * c.ny + j) * c.nz + k;
        const bool in_box = i >= b[0] && i < b[1] && j >= b[2] && j < b[3] && k >= b[4] && k < b[5];
        const int want = in_box && c.mat_disp[c.mat_id[q]] ? 1 : 0;
        if (seen[q] != want) fail("dispersive cell not covered exactly once", trial, i, j, k);
      }
  return static_cast<long long>(runs.size());
}

}  // namespace

int main() {
  std::mt19937 rng(5);
  long long items = 0, runs = 0;
  for (int trial = 0; trial < 160; ++trial) {
    const Compiled c = random_scene(rng, trial);
    for (int t = 0; t < kStepTileCount; ++t)
      for (int deferred = 0; deferred < 2; ++deferred) items += check_items(c, t, deferred != 0, trial);
  }
  for (int trial = 0; trial < 60; ++trial) runs += check_runs(rng, trial);
  if (bad) {
    std::printf("failures %d\n", bad);
    return 1;
  }
  std::printf("ok %lld %lld\n", items, runs);
  return 0;
}
