// Candidate launch shapes of the Euler / Navier-Stokes volume kernel per N+1, for the autotuner:
//   epb   elements per block;
//   lpw   lines per warp in the pair phase (0: lines contiguous in the thread index, needs N+1 | 32);
//   minb  resident blocks per SM the register allocation must allow (0: 2 up to 512 threads, else 1);
//   ownsm 1: a thread reads its own node's record from shared memory in every round instead of
//         holding it in registers (fewer registers, more shared-memory loads).
// Entry 0 of each list is the shape used before tuning.  All shapes of one N add the same terms in
// the same order (they agree to roundoff: the compiler's multiply-add fusion may differ between
// instantiations); they differ in occupancy, idle lanes, register spills and shared-memory traffic.
#pragma once

namespace fluxo {

struct VolShapeId {
  int epb, lpw, minb, ownsm;
};

constexpr int kVolShapeMax = 3;

// kVolShapes[NP][i]; an entry with epb 0 ends a list
constexpr VolShapeId kVolShapes[10][kVolShapeMax] = {
    {{0, 0, 0, 0}, {0, 0, 0, 0}, {0, 0, 0, 0}},    // NP 0 (unused)
    {{0, 0, 0, 0}, {0, 0, 0, 0}, {0, 0, 0, 0}},    // NP 1 (unused)
    {{32, 0, 0, 0}, {16, 0, 0, 0}, {0, 0, 0, 0}},  // NP 2: 256 / 128 threads
    {{8, 10, 0, 0}, {8, 8, 0, 0}, {4, 8, 0, 0}},   // NP 3: 256 / 512 / 256 threads
    {{4, 0, 0, 0}, {8, 0, 0, 0}, {2, 0, 0, 0}},    // NP 4: 256 / 512 / 128 threads
    {{2, 6, 0, 0}, {2, 4, 0, 0}, {1, 4, 0, 0}},    // NP 5: 320 / 448 / 224 threads
    {{1, 5, 0, 0}, {1, 4, 0, 0}, {1, 4, 0, 1}},    // NP 6: 256 / 288 / 288 threads
    {{1, 4, 0, 0}, {1, 4, 1, 0}, {1, 4, 0, 1}},    // NP 7: 416 threads; 1-block registers; own record in smem
    {{1, 0, 0, 0}, {1, 0, 1, 0}, {1, 0, 0, 1}},    // NP 8: 512 threads; 1-block registers; own record in smem
    {{1, 3, 0, 1}, {0, 0, 0, 0}, {0, 0, 0, 0}},    // NP 9: 864 threads
};

constexpr int vol_shape_count(int NP) {
  int c = 0;
  while (NP >= 0 && NP < 10 && c < kVolShapeMax && kVolShapes[NP][c].epb > 0) ++c;
  return c;
}

}  // namespace fluxo
