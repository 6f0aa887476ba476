// Host-side setup helpers shared by the C ABI implementation.
#pragma once
#include <vector>

namespace fluxo {
namespace host {
void flip_pq(int N, int p, int q, int flip, int& a, int& b);
void side_to_vol(int N, int l, int p, int q, int flip, int side, int* ijk);
void box_connectivity(const int* nElemsXYZ, int N, std::vector<int>& S2E, std::vector<int>& E2S);
}  // namespace host
}  // namespace fluxo
