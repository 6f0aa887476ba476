// Index arithmetic between volume nodes and face points with the reference's conventions
// (src/mesh/mappings.f90:262-464, CGNS local sides, flips 0..4), usable on host and device so the
// kernels need no lookup tables in global memory.
//   side_node: volume node (i + NP(j + NP k)) of face point (p,q) of local side s seen with flip
//              `flip` (the reference's S2V(:,0,p,q,flip,s)).
//   node_side_point: the inverse for a node on local side s of an element whose side is stored
//              with flip `flip`: the point index p + NP q in the master frame.
#pragma once

#if defined(__CUDACC__)
#define FLUXO_HD __host__ __device__ __forceinline__
#else
#define FLUXO_HD inline
#endif

namespace fluxo {

FLUXO_HD void flip_to_local(int N, int p, int q, int flip, int& a, int& b) {
  switch (flip) {
    case 0: a = p; b = q; return;
    case 1: a = q; b = p; return;
    case 2: a = N - p; b = q; return;
    case 3: a = N - q; b = N - p; return;
    default: a = p; b = N - q; return;
  }
}

FLUXO_HD int side_node(int N, int p, int q, int flip, int s) {
  int a, b, i, j, k;
  flip_to_local(N, p, q, flip, a, b);
  switch (s) {
    case 5: i = 0; j = b; k = a; break;          // XI_MINUS
    case 3: i = N; j = a; k = b; break;          // XI_PLUS
    case 2: i = a; j = 0; k = b; break;          // ETA_MINUS
    case 4: i = N - a; j = N; k = b; break;      // ETA_PLUS
    case 1: i = b; j = a; k = 0; break;          // ZETA_MINUS
    default: i = a; j = b; k = N; break;         // ZETA_PLUS
  }
  return i + (N + 1) * (j + (N + 1) * k);
}

FLUXO_HD int node_side_point(int N, int s, int flip, int i, int j, int k) {
  int a, b;  // the side's local (flipped) coordinates of node (i,j,k)
  switch (s) {
    case 5: a = k; b = j; break;
    case 3: a = j; b = k; break;
    case 2: a = i; b = k; break;
    case 4: a = N - i; b = k; break;
    case 1: a = j; b = i; break;
    default: a = i; b = j; break;
  }
  int p, q;  // invert flip_to_local
  switch (flip) {
    case 0: p = a; q = b; break;
    case 1: p = b; q = a; break;
    case 2: p = N - a; q = b; break;
    case 3: p = N - b; q = N - a; break;
    default: p = a; q = N - b; break;
  }
  return p + (N + 1) * q;
}

}  // namespace fluxo
