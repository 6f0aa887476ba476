// Host-side setup helpers shared by the C ABI implementation.
#pragma once
#include <string>
#include <vector>

namespace fluxo {
namespace host {
void flip_pq(int N, int p, int q, int flip, int& a, int& b);
void side_to_vol(int N, int l, int p, int q, int flip, int side, int* ijk);
void box_connectivity(const int* nElemsXYZ, int N, std::vector<int>& S2E, std::vector<int>& E2S);
// The reference's mesh arrays (Fortran layouts, 1-based ids, inner sides only) in the device
// layouts: s2e [side][5] with 0-based elements, e2s [elem][6][2] with 0-based sides, metrics
// [elem][9][node], face geometry [side][10][pt].  False (and a message) for out-of-range entries.
bool repack_mesh(int N, int nElems, int nSides, const int* S2E, const int* E2S, const double* Mf, const double* Mg,
                 const double* Mh, const double* NormVec, const double* TangVec1, const double* TangVec2,
                 const double* SurfElem, std::vector<int>& s2e, std::vector<int>& e2s, std::vector<double>& met,
                 std::vector<double>& geo, std::string& err);
}  // namespace host
}  // namespace fluxo
