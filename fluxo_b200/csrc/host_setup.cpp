// Host-side setup of the product (no GPU): side/volume index maps, a periodic hexahedral box
// with optional curved (NGeo) deformation, its curl-form metrics and surface metrics, and the
// initial states of the reference's exact functions.  This stands in for the reference's
// InitMesh / CalcMetrics (src/mesh/mesh.f90:89-296, src/mesh/metrics.f90:78-484), which read a
// HOPR HDF5 mesh; the arrays it produces have the reference layouts of include/fluxo_gpu.h.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <stdexcept>
#include <vector>

#include "../../include/fluxo_gpu.h"
#include "host_basis.h"
#include "host_setup.h"

namespace fluxo {
// fluxo_gpu.cu: the message that fluxo_gpu_last_error(NULL, ...) returns (returns `code`)
int record_unbound_error(int code, const std::string& msg);

namespace host {

// Side <-> volume index maps with the reference's conventions (src/mesh/mappings.f90:262-464):
// flip maps master (p,q) to slave coordinates; CGNS orientation of each local side.
void flip_pq(int N, int p, int q, int flip, int& a, int& b) {
  switch (flip) {
    case 0: a = p; b = q; return;
    case 1: a = q; b = p; return;
    case 2: a = N - p; b = q; return;
    case 3: a = N - q; b = N - p; return;
    default: a = p; b = N - q; return;
  }
}

void side_to_vol(int N, int l, int p, int q, int flip, int side, int* ijk) {
  int a, b;
  flip_pq(N, p, q, flip, a, b);
  switch (side) {
    case 5: ijk[0] = l; ijk[1] = b; ijk[2] = a; return;          // XI_MINUS
    case 3: ijk[0] = N - l; ijk[1] = a; ijk[2] = b; return;      // XI_PLUS
    case 2: ijk[0] = a; ijk[1] = l; ijk[2] = b; return;          // ETA_MINUS
    case 4: ijk[0] = N - a; ijk[1] = N - l; ijk[2] = b; return;  // ETA_PLUS
    case 1: ijk[0] = b; ijk[1] = a; ijk[2] = l; return;          // ZETA_MINUS
    default: ijk[0] = a; ijk[1] = b; ijk[2] = N - l; return;     // ZETA_PLUS
  }
}

namespace {

// tensor-product interpolation of `dim` interleaved fields from (ni)^3 to (no)^3 nodes, V is no x ni
void tp_interp(int dim, int ni, int no, const std::vector<double>& V, const double* in, double* out) {
  std::vector<double> a((size_t)dim * no * ni * ni, 0.), b((size_t)dim * no * no * ni, 0.);
  for (int k = 0; k < ni; ++k)
    for (int j = 0; j < ni; ++j)
      for (int o = 0; o < no; ++o)
        for (int i = 0; i < ni; ++i) {
          const double v = V[(size_t)o * ni + i];
          for (int d = 0; d < dim; ++d) a[d + dim * (o + no * (j + ni * k))] += v * in[d + dim * (i + ni * (j + ni * k))];
        }
  for (int k = 0; k < ni; ++k)
    for (int o = 0; o < no; ++o)
      for (int j = 0; j < ni; ++j) {
        const double v = V[(size_t)o * ni + j];
        for (int i = 0; i < no; ++i)
          for (int d = 0; d < dim; ++d) b[d + dim * (i + no * (o + no * k))] += v * a[d + dim * (i + no * (j + ni * k))];
      }
  std::fill(out, out + (size_t)dim * no * no * no, 0.);
  for (int o = 0; o < no; ++o)
    for (int k = 0; k < ni; ++k) {
      const double v = V[(size_t)o * ni + k];
      for (int j = 0; j < no; ++j)
        for (int i = 0; i < no; ++i)
          for (int d = 0; d < dim; ++d) out[d + dim * (i + no * (j + no * o))] += v * b[d + dim * (i + no * (j + no * k))];
    }
}

// derivative along reference direction `dir` of `dim` interleaved fields on n^3 nodes
void tp_deriv(int dim, int n, const std::vector<double>& D, int dir, const double* in, double* out) {
  for (int k = 0; k < n; ++k)
    for (int j = 0; j < n; ++j)
      for (int i = 0; i < n; ++i) {
        const int me = dir == 0 ? i : (dir == 1 ? j : k);
        for (int d = 0; d < dim; ++d) {
          double s = 0.;
          for (int l = 0; l < n; ++l) {
            const int ii = dir == 0 ? l : i, jj = dir == 1 ? l : j, kk = dir == 2 ? l : k;
            s += D[(size_t)me * n + l] * in[d + dim * (ii + n * (jj + n * kk))];
          }
          out[d + dim * (i + n * (j + n * k))] = s;
        }
      }
}

const int kNormalDir[7] = {0, 3, 2, 1, 2, 1, 3};  // src/mesh/mesh_vars.f90:91-93
const int kTangDir[7] = {0, 1, 3, 2, 3, 2, 1};
const double kNormalSign[7] = {0, -1., -1., 1., 1., -1., 1.};

}  // namespace

void box_connectivity(const int* ne, int N, std::vector<int>& S2E, std::vector<int>& E2S) {
  const int nx = ne[0], ny = ne[1], nz = ne[2];
  const int nElems = nx * ny * nz, nSides = 3 * nElems, n = N + 1;
  S2E.assign((size_t)5 * nSides, -1);
  E2S.assign((size_t)12 * nElems, 0);
  auto eid = [&](int x, int y, int z) { return ((z + nz) % nz) * nx * ny + ((y + ny) % ny) * nx + ((x + nx) % nx); };
  std::vector<int> owner((size_t)6 * nElems, 0);
  int next = 0;
  for (int e = 0; e < nElems; ++e) {
    const int ix = e % nx, iy = (e / nx) % ny, iz = e / (nx * ny);
    for (int s = 1; s <= 6; ++s) {
      if (owner[(size_t)6 * e + s - 1]) continue;
      int nb, nbs;
      switch (s) {
        case 5: nb = eid(ix - 1, iy, iz); nbs = 3; break;
        case 3: nb = eid(ix + 1, iy, iz); nbs = 5; break;
        case 2: nb = eid(ix, iy - 1, iz); nbs = 4; break;
        case 4: nb = eid(ix, iy + 1, iz); nbs = 2; break;
        case 1: nb = eid(ix, iy, iz - 1); nbs = 6; break;
        default: nb = eid(ix, iy, iz + 1); nbs = 1; break;
      }
      const int sid = ++next;
      owner[(size_t)6 * e + s - 1] = sid;
      owner[(size_t)6 * nb + nbs - 1] = sid;
      // slave flip: the one that maps every master face node onto the same global lattice node
      auto lat = [&](int el, const int* ijk, long* g) {
        const int x = el % nx, y = (el / nx) % ny, z = el / (nx * ny);
        g[0] = ((long)x * N + ijk[0]) % ((long)nx * N);
        g[1] = ((long)y * N + ijk[1]) % ((long)ny * N);
        g[2] = ((long)z * N + ijk[2]) % ((long)nz * N);
      };
      int flip = -1;
      for (int f = 1; f <= 4 && flip < 0; ++f) {
        bool ok = true;
        for (int q = 0; q < n && ok; ++q)
          for (int p = 0; p < n && ok; ++p) {
            int a[3], b[3];
            long ga[3], gb[3];
            side_to_vol(N, 0, p, q, 0, s, a);
            side_to_vol(N, 0, p, q, f, nbs, b);
            lat(e, a, ga);
            lat(nb, b, gb);
            ok = ga[0] == gb[0] && ga[1] == gb[1] && ga[2] == gb[2];
          }
        if (ok) flip = f;
      }
      if (flip < 0) throw std::runtime_error("box_connectivity: no flip");
      int* se = &S2E[(size_t)5 * (sid - 1)];
      se[0] = e + 1; se[1] = nb + 1; se[2] = s; se[3] = nbs; se[4] = flip;
      E2S[(size_t)2 * (6 * e + s - 1)] = sid;
      E2S[(size_t)2 * (6 * e + s - 1) + 1] = 0;
      E2S[(size_t)2 * (6 * nb + nbs - 1)] = sid;
      E2S[(size_t)2 * (6 * nb + nbs - 1) + 1] = flip;
    }
  }
  if (next != nSides) throw std::runtime_error("box_connectivity: side count");
}

// Node coordinates NodeCoords(3,0:NGeo,0:NGeo,0:NGeo,nElems) of the periodic box on equidistant points,
// deformed by X_d += amp * prod_e sin(2 pi (x_e - c_e) / L_e) (which keeps the box periodic).
std::vector<double> box_nodes(const int* ne, const double* xmin, const double* xmax, int NGeo, double amp) {
  const int nx = ne[0], ny = ne[1], nz = ne[2], nElems = nx * ny * nz, ng = NGeo + 1;
  const double L[3] = {xmax[0] - xmin[0], xmax[1] - xmin[1], xmax[2] - xmin[2]};
  const double c[3] = {0.5 * (xmax[0] + xmin[0]), 0.5 * (xmax[1] + xmin[1]), 0.5 * (xmax[2] + xmin[2])};
  const double h[3] = {L[0] / nx, L[1] / ny, L[2] / nz};
  std::vector<double> X((size_t)3 * ng * ng * ng * nElems);
  for (int e = 0; e < nElems; ++e) {
    const int ix = e % nx, iy = (e / nx) % ny, iz = e / (nx * ny);
    double* Xe = &X[(size_t)3 * ng * ng * ng * e];
    for (int k = 0; k < ng; ++k)
      for (int j = 0; j < ng; ++j)
        for (int i = 0; i < ng; ++i) {
          const double xs[3] = {xmin[0] + h[0] * (ix + (double)i / NGeo), xmin[1] + h[1] * (iy + (double)j / NGeo),
                                xmin[2] + h[2] * (iz + (double)k / NGeo)};
          double f = amp;
          if (f != 0.)
            for (int d = 0; d < 3; ++d) f *= std::sin(2. * M_PI * (xs[d] - c[d]) / L[d]);
          for (int d = 0; d < 3; ++d) Xe[3 * (i + ng * (j + ng * k)) + d] = xs[d] + f;
        }
  }
  return X;
}

// LGL nodes (CalcMetrics / CalcSurfMetrics, metrics.f90:78-440) from node coordinates of degree NGeo on
// equidistant (nodesGL false) or Gauss-Lobatto points.
void nodes_geometry(int N, int nElems, int NGeo, bool nodesGL, const double* NodeCoords, const std::vector<int>& E2S,
                    double* Mf, double* Mg, double* Mh, double* sJ, double* NormVec, double* TangVec1,
                    double* TangVec2, double* SurfElem, double* Elem_xGP) {
  const int n = N + 1, ng = NGeo + 1, NR = 3 * NGeo, nr = NR + 1;
  const size_t nv = (size_t)n * n * n;
  LGLBasis bN(N);
  std::vector<double> xeq(ng), xg, wg, xr, wr;
  lgl(NGeo, xg, wg);
  for (int i = 0; i < ng; ++i) xeq[i] = nodesGL ? xg[i] : 2. * i / NGeo - 1.;
  lgl(NR, xr, wr);
  const std::vector<double> V_eq_g = interp_matrix(xeq, xg);
  const std::vector<double> V_g_N = interp_matrix(xg, bN.x);
  const std::vector<double> V_g_r = interp_matrix(xg, xr);
  std::vector<double> V_r_N;
  if (NR > N) V_r_N = modal_projection(xr, bN.x);
  else V_r_N = interp_matrix(xr, bN.x);
  const std::vector<double> Dg = deriv_matrix(xg);
#pragma omp parallel for schedule(dynamic, 16)
  for (int e = 0; e < nElems; ++e) {
    std::vector<double> Xg(3 * ng * ng * ng), XN(3 * nv), dXg(9 * ng * ng * ng), tmp(3 * ng * ng * ng);
    tp_interp(3, ng, ng, V_eq_g, NodeCoords + (size_t)3 * ng * ng * ng * e, Xg.data());
    tp_interp(3, ng, n, V_g_N, Xg.data(), XN.data());
    std::copy(XN.begin(), XN.end(), Elem_xGP + 3 * nv * e);
    // dXg[dir][node][coord]: derivative of the coordinates along reference direction dir (NGeo nodes)
    for (int dir = 0; dir < 3; ++dir) {
      tp_deriv(3, ng, Dg, dir, Xg.data(), tmp.data());
      for (int z = 0; z < ng * ng * ng; ++z)
        for (int d = 0; d < 3; ++d) dXg[9 * z + 3 * dir + d] = tmp[3 * z + d];
    }
    // Jacobian determinant at 3*NGeo, then projected (or interpolated) to N
    std::vector<double> dXr((size_t)9 * nr * nr * nr), detr((size_t)nr * nr * nr), detN(nv);
    tp_interp(9, ng, nr, V_g_r, dXg.data(), dXr.data());
    for (int z = 0; z < nr * nr * nr; ++z) {
      const double* a = &dXr[9 * z];  // a[3*dir + coord] = dX_coord/dxi_dir
      const double* t = a;
      const double* u = a + 3;
      const double* w = a + 6;
      detr[z] = t[0] * (u[1] * w[2] - u[2] * w[1]) - t[1] * (u[0] * w[2] - u[2] * w[0]) + t[2] * (u[0] * w[1] - u[1] * w[0]);
    }
    if (NR == N) std::copy(detr.begin(), detr.end(), detN.begin());
    else tp_interp(1, nr, n, V_r_N, detr.data(), detN.data());
    for (size_t z = 0; z < nv; ++z) sJ[nv * e + z] = 1. / detN[z];
    // coordinate derivatives on the N nodes
    std::vector<double> dXN((size_t)9 * nv), tN(3 * nv);
    if (N >= NGeo) {
      tp_interp(9, ng, n, V_g_N, dXg.data(), dXN.data());
    } else {
      for (int dir = 0; dir < 3; ++dir) {
        tp_deriv(3, n, bN.D, dir, XN.data(), tN.data());
        for (size_t z = 0; z < nv; ++z)
          for (int d = 0; d < 3; ++d) dXN[9 * z + 3 * dir + d] = tN[3 * z + d];
      }
    }
    // curl form: Ja^i_c = -(curl_xi R_c)_i with R_c(dir) = 1/2 (X_{c+2} dX_{c+1}/dxi_dir - X_{c+1} dX_{c+2}/dxi_dir)
    std::vector<double> R((size_t)9 * nv), dR((size_t)9 * nv), Ja((size_t)9 * nv, 0.);  // R[9*z + 3*dir + c]
    for (size_t z = 0; z < nv; ++z)
      for (int dir = 0; dir < 3; ++dir)
        for (int cc = 0; cc < 3; ++cc) {
          const int c1 = (cc + 1) % 3, c2 = (cc + 2) % 3;
          R[9 * z + 3 * dir + cc] = 0.5 * (XN[3 * z + c2] * dXN[9 * z + 3 * dir + c1] - XN[3 * z + c1] * dXN[9 * z + 3 * dir + c2]);
        }
    // Ja(i,c) += d/dxi_{i+2} R(i+1,c) - d/dxi_{i+1} R(i+2,c)
    for (int dd = 0; dd < 3; ++dd) {
      tp_deriv(9, n, bN.D, dd, R.data(), dR.data());  // dR[.. 3*dir + c] = d/dxi_dd R(dir,c)
      for (size_t z = 0; z < nv; ++z)
        for (int i = 0; i < 3; ++i)
          for (int cc = 0; cc < 3; ++cc) {
            if (dd == (i + 2) % 3) Ja[9 * z + 3 * i + cc] += dR[9 * z + 3 * ((i + 1) % 3) + cc];
            if (dd == (i + 1) % 3) Ja[9 * z + 3 * i + cc] -= dR[9 * z + 3 * ((i + 2) % 3) + cc];
          }
    }
    for (size_t z = 0; z < nv; ++z)
      for (int cc = 0; cc < 3; ++cc) {
        Mf[3 * (nv * e + z) + cc] = Ja[9 * z + 0 + cc];
        Mg[3 * (nv * e + z) + cc] = Ja[9 * z + 3 + cc];
        Mh[3 * (nv * e + z) + cc] = Ja[9 * z + 6 + cc];
      }
    // surface metrics of the master sides (CalcSurfMetrics / SurfMetricsFromJa)
    for (int s = 1; s <= 6; ++s) {
      const int sid = E2S[(size_t)2 * (6 * e + s - 1)], flip = E2S[(size_t)2 * (6 * e + s - 1) + 1];
      if (flip != 0) continue;
      const int nd = kNormalDir[s] - 1, td = kTangDir[s] - 1;
      for (int q = 0; q < n; ++q)
        for (int p = 0; p < n; ++p) {
          int ijk[3];
          side_to_vol(N, 0, p, q, 0, s, ijk);
          const size_t z = ijk[0] + n * (ijk[1] + (size_t)n * ijk[2]);
          const double* jn = &Ja[9 * z + 3 * nd];
          const double* jt = &Ja[9 * z + 3 * td];
          const size_t fi = p + n * (q + (size_t)n * (sid - 1));
          const double se = std::sqrt(jn[0] * jn[0] + jn[1] * jn[1] + jn[2] * jn[2]);
          double nv3[3], t1[3];
          for (int d = 0; d < 3; ++d) nv3[d] = kNormalSign[s] * jn[d] / se;
          const double dot = jt[0] * nv3[0] + jt[1] * nv3[1] + jt[2] * nv3[2];
          for (int d = 0; d < 3; ++d) t1[d] = jt[d] - dot * nv3[d];
          const double tn = std::sqrt(t1[0] * t1[0] + t1[1] * t1[1] + t1[2] * t1[2]);
          for (int d = 0; d < 3; ++d) t1[d] /= tn;
          SurfElem[fi] = se;
          for (int d = 0; d < 3; ++d) {
            NormVec[3 * fi + d] = nv3[d];
            TangVec1[3 * fi + d] = t1[d];
          }
          TangVec2[3 * fi + 0] = nv3[1] * t1[2] - nv3[2] * t1[1];
          TangVec2[3 * fi + 1] = nv3[2] * t1[0] - nv3[0] * t1[2];
          TangVec2[3 * fi + 2] = nv3[0] * t1[1] - nv3[1] * t1[0];
        }
    }
  }
}

// Gauss nodes (CalcMetrics / CalcSurfMetrics with NodeType 'GAUSS', metrics.f90:78-440): the coordinates,
// their derivatives and the curl-form metric terms on the Gauss-Lobatto points of degree N, then
// interpolated to the Gauss nodes (Vdm_GLN_N); the Jacobian through 3*NGeo Gauss points, projected to N;
// the side quantities from the Gauss-Lobatto metric terms of the side interpolated to the side's Gauss
// points, SurfMetrics (the normal metric term) for every side in the master's point order.
void nodes_geometry_gauss(int N, int nElems, int NGeo, bool nodesGL, const double* NodeCoords,
                          const std::vector<int>& E2S, double* Mf, double* Mg, double* Mh, double* sJ,
                          double* NormVec, double* TangVec1, double* TangVec2, double* SurfElem, double* Elem_xGP,
                          double* SurfMetrics) {
  const int n = N + 1, ng = NGeo + 1, NR = 3 * NGeo, nr = NR + 1;
  const size_t nv = (size_t)n * n * n;
  GaussBasis bG(N);
  std::vector<double> xeq(ng), xg, wg, xr, wr, xGL, wGL;
  lgl(NGeo, xg, wg);
  for (int i = 0; i < ng; ++i) xeq[i] = nodesGL ? xg[i] : 2. * i / NGeo - 1.;
  gauss(NR, xr, wr);
  lgl(N, xGL, wGL);
  const std::vector<double> V_eq_g = interp_matrix(xeq, xg);
  const std::vector<double> V_g_GL = interp_matrix(xg, xGL);
  const std::vector<double> V_GL_N = interp_matrix(xGL, bG.x);
  const std::vector<double> V_g_r = interp_matrix(xg, xr);
  std::vector<double> V_r_N;
  if (NR > N) V_r_N = modal_projection(xr, bG.x);
  else if (NR < N) V_r_N = interp_matrix(xr, bG.x);
  const std::vector<double> Dg = deriv_matrix(xg), DGL = deriv_matrix(xGL);
#pragma omp parallel for schedule(dynamic, 16)
  for (int e = 0; e < nElems; ++e) {
    std::vector<double> Xg(3 * ng * ng * ng), XGL(3 * nv), dXg(9 * ng * ng * ng), tmp(3 * ng * ng * ng);
    tp_interp(3, ng, ng, V_eq_g, NodeCoords + (size_t)3 * ng * ng * ng * e, Xg.data());
    tp_interp(3, ng, n, V_g_GL, Xg.data(), XGL.data());
    tp_interp(3, n, n, V_GL_N, XGL.data(), Elem_xGP + 3 * nv * e);
    for (int dir = 0; dir < 3; ++dir) {
      tp_deriv(3, ng, Dg, dir, Xg.data(), tmp.data());
      for (int z = 0; z < ng * ng * ng; ++z)
        for (int d = 0; d < 3; ++d) dXg[9 * z + 3 * dir + d] = tmp[3 * z + d];
    }
    std::vector<double> dXr((size_t)9 * nr * nr * nr), detr((size_t)nr * nr * nr), detN(nv);
    tp_interp(9, ng, nr, V_g_r, dXg.data(), dXr.data());
    for (int z = 0; z < nr * nr * nr; ++z) {
      const double* t = &dXr[9 * z];
      const double* u = t + 3;
      const double* w = t + 6;
      detr[z] = t[0] * (u[1] * w[2] - u[2] * w[1]) - t[1] * (u[0] * w[2] - u[2] * w[0]) + t[2] * (u[0] * w[1] - u[1] * w[0]);
    }
    if (NR == N) std::copy(detr.begin(), detr.end(), detN.begin());
    else tp_interp(1, nr, n, V_r_N, detr.data(), detN.data());
    for (size_t z = 0; z < nv; ++z) sJ[nv * e + z] = 1. / detN[z];
    std::vector<double> dXN((size_t)9 * nv), tN(3 * nv);
    if (N >= NGeo) {
      tp_interp(9, ng, n, V_g_GL, dXg.data(), dXN.data());
    } else {
      for (int dir = 0; dir < 3; ++dir) {
        tp_deriv(3, n, DGL, dir, XGL.data(), tN.data());
        for (size_t z = 0; z < nv; ++z)
          for (int d = 0; d < 3; ++d) dXN[9 * z + 3 * dir + d] = tN[3 * z + d];
      }
    }
    std::vector<double> R((size_t)9 * nv), dR((size_t)9 * nv), Ja((size_t)9 * nv, 0.), JaG((size_t)9 * nv);
    for (size_t z = 0; z < nv; ++z)
      for (int dir = 0; dir < 3; ++dir)
        for (int cc = 0; cc < 3; ++cc) {
          const int c1 = (cc + 1) % 3, c2 = (cc + 2) % 3;
          R[9 * z + 3 * dir + cc] = 0.5 * (XGL[3 * z + c2] * dXN[9 * z + 3 * dir + c1] - XGL[3 * z + c1] * dXN[9 * z + 3 * dir + c2]);
        }
    for (int dd = 0; dd < 3; ++dd) {
      tp_deriv(9, n, DGL, dd, R.data(), dR.data());
      for (size_t z = 0; z < nv; ++z)
        for (int i = 0; i < 3; ++i)
          for (int cc = 0; cc < 3; ++cc) {
            if (dd == (i + 2) % 3) Ja[9 * z + 3 * i + cc] += dR[9 * z + 3 * ((i + 1) % 3) + cc];
            if (dd == (i + 1) % 3) Ja[9 * z + 3 * i + cc] -= dR[9 * z + 3 * ((i + 2) % 3) + cc];
          }
    }
    tp_interp(9, n, n, V_GL_N, Ja.data(), JaG.data());
    for (size_t z = 0; z < nv; ++z)
      for (int cc = 0; cc < 3; ++cc) {
        Mf[3 * (nv * e + z) + cc] = JaG[9 * z + 0 + cc];
        Mg[3 * (nv * e + z) + cc] = JaG[9 * z + 3 + cc];
        Mh[3 * (nv * e + z) + cc] = JaG[9 * z + 6 + cc];
      }
    // sides: the Gauss-Lobatto boundary slice of Ja (tangential volume indices in increasing order)
    // interpolated to the side's Gauss points
    std::vector<double> sl((size_t)9 * n * n), b1((size_t)9 * n * n), JaF((size_t)9 * n * n);
    for (int s = 1; s <= 6; ++s) {
      const int sid = E2S[(size_t)2 * (6 * e + s - 1)], flip = E2S[(size_t)2 * (6 * e + s - 1) + 1];
      for (int b = 0; b < n; ++b)
        for (int a = 0; a < n; ++a) {
          int i, j, k;
          switch (s) {
            case 5: i = 0; j = a; k = b; break;
            case 3: i = N; j = a; k = b; break;
            case 2: i = a; j = 0; k = b; break;
            case 4: i = a; j = N; k = b; break;
            case 1: i = a; j = b; k = 0; break;
            default: i = a; j = b; k = N; break;
          }
          for (int q = 0; q < 9; ++q) sl[q + 9 * (a + n * b)] = Ja[9 * (i + n * (j + (size_t)n * k)) + q];
        }
      std::fill(b1.begin(), b1.end(), 0.);
      std::fill(JaF.begin(), JaF.end(), 0.);
      for (int b = 0; b < n; ++b)
        for (int ao = 0; ao < n; ++ao)
          for (int a = 0; a < n; ++a)
            for (int q = 0; q < 9; ++q) b1[q + 9 * (ao + n * b)] += V_GL_N[(size_t)ao * n + a] * sl[q + 9 * (a + n * b)];
      for (int bo = 0; bo < n; ++bo)
        for (int b = 0; b < n; ++b)
          for (int a = 0; a < n; ++a)
            for (int q = 0; q < 9; ++q) JaF[q + 9 * (a + n * bo)] += V_GL_N[(size_t)bo * n + b] * b1[q + 9 * (a + n * b)];
      const int nd = kNormalDir[s] - 1, td = kTangDir[s] - 1;
      for (int q = 0; q < n; ++q)
        for (int p = 0; p < n; ++p) {
          int ijk[3];
          side_to_vol(N, 0, p, q, 0, s, ijk);  // the element's own (CGNS) frame of the side
          const int a = (s == 5 || s == 3) ? ijk[1] : ijk[0];
          const int b = (s == 1 || s == 6) ? ijk[1] : ijk[2];
          const double* J = &JaF[9 * (a + n * b)];
          const double* jn = J + 3 * nd;
          const double* jt = J + 3 * td;
          int pm, qm;
          flip_pq(N, p, q, flip, pm, qm);  // FS2M: the master side's point (the flips are involutions)
          double* SM = SurfMetrics + 3 * ((size_t)pm + n * ((size_t)qm + n * ((size_t)(s - 1) + 6 * (size_t)e)));
          for (int d = 0; d < 3; ++d) SM[d] = jn[d];
          if (flip != 0) continue;
          const size_t fi = p + n * (q + (size_t)n * (sid - 1));
          const double se = std::sqrt(jn[0] * jn[0] + jn[1] * jn[1] + jn[2] * jn[2]);
          double nv3[3], t1[3];
          for (int d = 0; d < 3; ++d) nv3[d] = kNormalSign[s] * jn[d] / se;
          const double dot = jt[0] * nv3[0] + jt[1] * nv3[1] + jt[2] * nv3[2];
          for (int d = 0; d < 3; ++d) t1[d] = jt[d] - dot * nv3[d];
          const double tn = std::sqrt(t1[0] * t1[0] + t1[1] * t1[1] + t1[2] * t1[2]);
          for (int d = 0; d < 3; ++d) t1[d] /= tn;
          SurfElem[fi] = se;
          for (int d = 0; d < 3; ++d) {
            NormVec[3 * fi + d] = nv3[d];
            TangVec1[3 * fi + d] = t1[d];
          }
          TangVec2[3 * fi + 0] = nv3[1] * t1[2] - nv3[2] * t1[1];
          TangVec2[3 * fi + 1] = nv3[2] * t1[0] - nv3[0] * t1[2];
          TangVec2[3 * fi + 2] = nv3[0] * t1[1] - nv3[1] * t1[0];
        }
    }
  }
}

// Connectivity of a HOPR mesh from the arrays of its file (ReadMesh, mesh_readin.f90:295-445;
// setLocalSideIDs, prepare_mesh.f90:59-215; fillMeshInfo, prepare_mesh.f90:662-710), for one process.
// ElemInfo(6,nElems): ELEM_FirstSideInd (row 3) is the 0-based offset of the element's six SideInfo
// records.  SideInfo(5,nSideInfo): SIDE_Type, SIDE_ID (> 0: the oriented side, flip 0; < 0: flip
// MOD(SIDE_Flip,10)), SIDE_nbElemID, SIDE_Flip, SIDE_BCID.  BCType(4,nBCs): BC_TYPE 1 (periodic) and
// 100 keep their connection.  Both records of a unique side are paired through |SIDE_ID|; side ids
// are handed out in element / local-side order as the reference does when every side is an inner
// side.  Mortar sides and sides of non-periodic boundaries are refused (the product's face kernels
// hold inner sides only).
bool hopr_connectivity(int nElems, const int* ElemInfo, int nSideInfo, const int* SideInfo, int nBCs,
                       const int* BCType, std::vector<int>& S2E, std::vector<int>& E2S, std::string& err) {
  const size_t nRec = 6 * (size_t)nElems;
  std::vector<int> uid(nRec), flip(nRec), nb(nRec);
  int maxUid = 0;
  for (int e = 0; e < nElems; ++e) {
    const int first = ElemInfo[6 * (size_t)e + 2];
    for (int ls = 0; ls < 6; ++ls) {
      const long row = (long)first + ls;
      if (row < 0 || row >= nSideInfo) { err = "ElemInfo: side offset out of range"; return false; }
      const int* r = SideInfo + 5 * row;
      if (r[0] < 0 || r[2] < 0) { err = "mortar sides are not supported"; return false; }
      if (r[4] != 0) {
        if (r[4] < 1 || r[4] > nBCs) { err = "SideInfo: BC index out of range"; return false; }
        const int type = BCType[4 * (size_t)(r[4] - 1)];
        if (type != 1 && type != 100) { err = "non-periodic boundary sides are not supported"; return false; }
      }
      if (r[2] == 0) { err = "boundary sides are not supported"; return false; }
      if (r[2] > nElems) { err = "SideInfo: neighbour element out of range"; return false; }
      const size_t a = 6 * (size_t)e + ls;
      uid[a] = r[1] > 0 ? r[1] : -r[1];
      flip[a] = r[1] > 0 ? 0 : r[3] % 10;
      if (uid[a] == 0 || flip[a] < 0 || flip[a] > 4) { err = "SideInfo: invalid side id or flip"; return false; }
      nb[a] = r[2] - 1;
      maxUid = std::max(maxUid, uid[a]);
    }
  }
  // pair the two records of every unique side
  std::vector<long> firstRec((size_t)maxUid + 1, -1), partner(nRec, -1);
  for (size_t a = 0; a < nRec; ++a) {
    long& f = firstRec[uid[a]];
    if (f < 0) { f = (long)a; continue; }
    if (f == -2 || partner[f] >= 0) { err = "a unique side with more than two element sides"; return false; }
    partner[f] = (long)a;
    partner[a] = f;
  }
  for (size_t a = 0; a < nRec; ++a) {
    if (partner[a] < 0) { err = "a side without a neighbour"; return false; }
    if (nb[a] != (int)(partner[a] / 6)) { err = "SideInfo: neighbour element does not hold the side"; return false; }
    if ((flip[a] == 0) == (flip[partner[a]] == 0)) { err = "a side needs one oriented (flip 0) element side"; return false; }
  }
  const int nSides = (int)(nRec / 2);
  S2E.assign((size_t)5 * nSides, -1);
  E2S.assign((size_t)2 * nRec, 0);
  std::vector<int> sid(nRec, 0);
  int next = 0;
  for (size_t a = 0; a < nRec; ++a) {
    if (!sid[a]) sid[a] = sid[partner[a]] = ++next;
    const int e = (int)(a / 6), ls = (int)(a % 6) + 1;
    E2S[2 * a] = sid[a];
    E2S[2 * a + 1] = flip[a];
    int* se = &S2E[(size_t)5 * (sid[a] - 1)];
    if (flip[a] == 0) { se[0] = e + 1; se[2] = ls; }
    else { se[1] = e + 1; se[3] = ls; se[4] = flip[a]; }
  }
  return true;
}

bool repack_mesh(int N, int nElems, int nSides, const int* S2E, const int* E2S, const double* Mf, const double* Mg,
                 const double* Mh, const double* NormVec, const double* TangVec1, const double* TangVec2,
                 const double* SurfElem, std::vector<int>& s2e, std::vector<int>& e2s, std::vector<double>& met,
                 std::vector<double>& geo, std::string& err) {
  const int NP = N + 1, NP3 = NP * NP * NP, NPT = NP * NP;
  s2e.assign((size_t)5 * nSides, 0);
  e2s.assign((size_t)12 * nElems, 0);
  for (int s = 0; s < nSides; ++s) {
    const int* a = S2E + 5 * (size_t)s;
    if (a[0] < 1 || a[0] > nElems || a[1] < 1 || a[1] > nElems || a[2] < 1 || a[2] > 6 || a[3] < 1 || a[3] > 6 ||
        a[4] < 1 || a[4] > 4) {
      err = "SideToElem entry out of range (only inner sides are supported)";
      return false;
    }
    s2e[5 * (size_t)s + 0] = a[0] - 1; s2e[5 * (size_t)s + 1] = a[1] - 1;
    s2e[5 * (size_t)s + 2] = a[2]; s2e[5 * (size_t)s + 3] = a[3]; s2e[5 * (size_t)s + 4] = a[4];
  }
  for (int e = 0; e < nElems; ++e)
    for (int ls = 0; ls < 6; ++ls) {
      const int sid = E2S[2 * (6 * (size_t)e + ls)], fl = E2S[2 * (6 * (size_t)e + ls) + 1];
      if (sid < 1 || sid > nSides || fl < 0 || fl > 4) {
        err = "ElemToSide out of range";
        return false;
      }
      e2s[2 * (6 * (size_t)e + ls)] = sid - 1;
      e2s[2 * (6 * (size_t)e + ls) + 1] = fl;
    }
  met.resize((size_t)9 * NP3 * nElems);
  geo.resize((size_t)10 * NPT * nSides);
  // element- and side-parallel: a large request (24^3 elements at N=7, 0.7 GB) is repacked while a
  // served batch keeps the GPU busy, and before the first step of a single solve
#pragma omp parallel for schedule(static)
  for (int e = 0; e < nElems; ++e)
    for (int d = 0; d < 3; ++d)
      for (int n = 0; n < NP3; ++n) {
        const size_t src = 3 * ((size_t)e * NP3 + n) + d;
        met[((size_t)e * 9 + d) * NP3 + n] = Mf[src];
        met[((size_t)e * 9 + 3 + d) * NP3 + n] = Mg[src];
        met[((size_t)e * 9 + 6 + d) * NP3 + n] = Mh[src];
      }
#pragma omp parallel for schedule(static)
  for (int s = 0; s < nSides; ++s)
    for (int p = 0; p < NPT; ++p) {
      const size_t src = (size_t)s * NPT + p;
      for (int d = 0; d < 3; ++d) {
        geo[((size_t)s * 10 + d) * NPT + p] = NormVec[3 * src + d];
        geo[((size_t)s * 10 + 3 + d) * NPT + p] = TangVec1[3 * src + d];
        geo[((size_t)s * 10 + 6 + d) * NPT + p] = TangVec2[3 * src + d];
      }
      geo[((size_t)s * 10 + 9) * NPT + p] = SurfElem[src];
    }
  return true;
}

}  // namespace host
}  // namespace fluxo

using namespace fluxo::host;

extern "C" int fluxo_host_box_sizes(const int* ne, int* nElems, int* nSides) {
  if (!ne || ne[0] < 1 || ne[1] < 1 || ne[2] < 1) return FLUXO_EINVAL_CFG;
  *nElems = ne[0] * ne[1] * ne[2];
  *nSides = 3 * *nElems;
  return FLUXO_OK;
}

extern "C" int fluxo_host_box_mesh(int N, const int* ne, const double* xmin, const double* xmax, int NGeo,
                                   double amp, int* SideToElem, int* ElemToSide, double* Mf, double* Mg, double* Mh,
                                   double* sJ, double* NormVec, double* TangVec1, double* TangVec2,
                                   double* SurfElem, double* Elem_xGP) {
  if (N < 1 || N > 8 || NGeo < 1 || !ne) return FLUXO_EINVAL_CFG;
  try {
    std::vector<int> S2E, E2S;
    box_connectivity(ne, N, S2E, E2S);
    std::copy(S2E.begin(), S2E.end(), SideToElem);
    std::copy(E2S.begin(), E2S.end(), ElemToSide);
    const std::vector<double> X = box_nodes(ne, xmin, xmax, NGeo, amp);
    nodes_geometry(N, ne[0] * ne[1] * ne[2], NGeo, false, X.data(), E2S, Mf, Mg, Mh, sJ, NormVec, TangVec1, TangVec2,
                   SurfElem, Elem_xGP);
  } catch (...) {
    return FLUXO_EINVAL_CFG;
  }
  return FLUXO_OK;
}

extern "C" int fluxo_host_box_mesh_gauss(int N, const int* ne, const double* xmin, const double* xmax, int NGeo,
                                         double amp, int* SideToElem, int* ElemToSide, double* Mf, double* Mg,
                                         double* Mh, double* sJ, double* NormVec, double* TangVec1, double* TangVec2,
                                         double* SurfElem, double* Elem_xGP, double* SurfMetrics) {
  if (N < 1 || N > 8 || NGeo < 1 || !ne || !SurfMetrics) return FLUXO_EINVAL_CFG;
  try {
    std::vector<int> S2E, E2S;
    box_connectivity(ne, N, S2E, E2S);
    std::copy(S2E.begin(), S2E.end(), SideToElem);
    std::copy(E2S.begin(), E2S.end(), ElemToSide);
    const std::vector<double> X = box_nodes(ne, xmin, xmax, NGeo, amp);
    nodes_geometry_gauss(N, ne[0] * ne[1] * ne[2], NGeo, false, X.data(), E2S, Mf, Mg, Mh, sJ, NormVec, TangVec1,
                         TangVec2, SurfElem, Elem_xGP, SurfMetrics);
  } catch (...) {
    return FLUXO_EINVAL_CFG;
  }
  return FLUXO_OK;
}

extern "C" int fluxo_host_hopr_mesh(int N, int node_type, int nElems, const int* ElemInfo, int nSideInfo,
                                    const int* SideInfo, int nBCs, const int* BCType, int NGeo, int mesh_nodes_gl,
                                    const double* NodeCoords, double mesh_scale, int use_curveds, int* SideToElem,
                                    int* ElemToSide, double* Mf, double* Mg, double* Mh, double* sJ, double* NormVec,
                                    double* TangVec1, double* TangVec2, double* SurfElem, double* Elem_xGP,
                                    double* SurfMetrics) {
  if (N < 1 || N > 8 || NGeo < 1 || nElems < 1 || !ElemInfo || !SideInfo || !NodeCoords || (nBCs > 0 && !BCType) ||
      (node_type != 1 && node_type != 2) || (node_type == 1 && !SurfMetrics))
    return FLUXO_EINVAL_CFG;
  try {
    std::vector<int> S2E, E2S;
    std::string err;
    if (!hopr_connectivity(nElems, ElemInfo, nSideInfo, SideInfo, nBCs, BCType, S2E, E2S, err))
      return fluxo::record_unbound_error(FLUXO_EINVAL_CFG, "fluxo_host_hopr_mesh: " + err);
    std::copy(S2E.begin(), S2E.end(), SideToElem);
    std::copy(E2S.begin(), E2S.end(), ElemToSide);
    // useCurveds = F keeps the eight corners (NGeo = 1); meshScale multiplies (mesh_readin.f90:466-481,
    // mesh.f90:233-236)
    const int ng = NGeo + 1;
    std::vector<double> X;
    int NG = NGeo;
    if (use_curveds) {
      X.assign(NodeCoords, NodeCoords + (size_t)3 * ng * ng * ng * nElems);
    } else {
      NG = 1;
      X.resize((size_t)24 * nElems);
      for (int e = 0; e < nElems; ++e)
        for (int c = 0; c < 8; ++c) {
          const int i = (c & 1) * NGeo, j = ((c >> 1) & 1) * NGeo, k = (c >> 2) * NGeo;
          for (int d = 0; d < 3; ++d)
            X[(size_t)24 * e + 3 * c + d] = NodeCoords[3 * (i + ng * (j + ng * (k + (size_t)ng * e))) + d];
        }
    }
    if (std::fabs(mesh_scale - 1.) > 1e-14)
      for (double& x : X) x *= mesh_scale;
    const bool gl = mesh_nodes_gl && use_curveds;
    if (node_type == 1)
      nodes_geometry_gauss(N, nElems, NG, gl, X.data(), E2S, Mf, Mg, Mh, sJ, NormVec, TangVec1, TangVec2, SurfElem,
                           Elem_xGP, SurfMetrics);
    else
      nodes_geometry(N, nElems, NG, gl, X.data(), E2S, Mf, Mg, Mh, sJ, NormVec, TangVec1, TangVec2, SurfElem,
                     Elem_xGP);
  } catch (...) {
    return FLUXO_EINVAL_CFG;
  }
  return FLUXO_OK;
}

extern "C" int fluxo_host_nodes(int N, int node_type, double* x, double* w) {
  if (N < 0 || N > 32 || !x || (node_type != 1 && node_type != 2)) return FLUXO_EINVAL_CFG;
  std::vector<double> xs, ws;
  if (node_type == 1) gauss(N, xs, ws);
  else lgl(N, xs, ws);
  std::copy(xs.begin(), xs.end(), x);
  if (w) std::copy(ws.begin(), ws.end(), w);
  return FLUXO_OK;
}

extern "C" int fluxo_host_exact_func(int func, double t, size_t np, const double* x, double kappa,
                                     const double* adv, double amp, const double* wave, double freq,
                                     const double* ref, double* U) {
  const double km1 = kappa - 1., skm1 = 1. / km1;
  for (size_t z = 0; z < np; ++z) {
    const double* X = x + 3 * z;
    double* u = U + 5 * z;
    double prim[5];
    switch (func) {
      case 1:  // constant state
        for (int v = 0; v < 5; ++v) prim[v] = ref[v];
        break;
      case 2: {  // density sine wave advected with AdvVel
        double arg = 0.;
        for (int d = 0; d < 3; ++d) arg += wave[d] * (X[d] - adv[d] * t);
        prim[0] = 1. + amp * std::sin(M_PI * arg);
        for (int d = 0; d < 3; ++d) prim[1 + d] = adv[d];
        prim[4] = 1.;
        break;
      }
      case 4: {  // manufactured solution rho = rho v_i = 2 + A sin(pi f (x+y+z-t)), rho E = rho^2
        const double r = 2. + amp * std::sin(M_PI * freq * (X[0] + X[1] + X[2] - t));
        u[0] = u[1] = u[2] = u[3] = r;
        u[4] = r * r;
        continue;
      }
      case 7: {  // Taylor-Green vortex, Mach 0.1
        prim[0] = 1.;
        prim[1] = std::sin(X[0]) * std::cos(X[1]) * std::cos(X[2]);
        prim[2] = -std::cos(X[0]) * std::sin(X[1]) * std::cos(X[2]);
        prim[3] = 0.;
        prim[4] = 100. / kappa + 1. / 16. * (std::cos(2 * X[0]) * std::cos(2. * X[2]) + 2. * std::cos(2. * X[1]) +
                                           2. * std::cos(2. * X[0]) + std::cos(2 * X[1]) * std::cos(2. * X[2]));
        break;
      }
      case 14: {  // soft Sedov-Taylor blast around IniCenter = 0 (its default), navierstokes/equation.f90:906-922
        const double r2 = std::sqrt(X[0] * X[0] + X[1] * X[1] + X[2] * X[2]);
        prim[0] = 1.; prim[1] = prim[2] = prim[3] = 0.; prim[4] = 1.;
        if (r2 <= 0.5 && r2 != 0.) {
          prim[0] = 1.3416149068323;
          for (int d = 0; d < 3; ++d) prim[1 + d] = 0.361538208967199 * X[d] / r2;
          prim[4] = 1.51333333333333;
        }
        break;
      }
      default:
        return FLUXO_EINVAL_CFG;
    }
    u[0] = prim[0];
    for (int d = 0; d < 3; ++d) u[1 + d] = prim[0] * prim[1 + d];
    u[4] = skm1 * prim[4] + 0.5 * (u[1] * prim[1] + u[2] * prim[2] + u[3] * prim[3]);
  }
  return FLUXO_OK;
}
