// Per-node records and symmetric two-point volume fluxes for the split-form volume kernel.
//
// Each volume node stores a record of the quantities its pair fluxes need (primitive variables,
// the logarithms of the log-averaged quantities, the metric terms of the three directions), so a
// pair evaluation does no logarithm and at most one division.  The fluxes are the reference's
// VolumeFluxAverageVec family (src/equation/navierstokes/flux_average.f90); results agree with
// the reference formulas to roundoff:
//  - the logarithmic mean LN_MEAN (flux_average.f90:1945-1965) keeps its series branch for
//    f^2 = ((b-a)/(b+a))^2 < 1e-4, written as 0.5 s^7 / (s^6 + s^4 d^2/3 + s^2 d^4/5 + d^6/7)
//    (s = a+b, d = b-a; identical to (a+b)*52.5/(105+35u+21u^2+15u^3)), and otherwise uses
//    (b-a)/(log b - log a) with per-node logarithms;
//  - every log mean is kept as a (numerator, denominator) pair and all divisions of one pair
//    flux are merged into a single reciprocal (rcp_nr).
#pragma once
#include "common.cuh"

namespace fluxo {

// Reciprocal of x > 0 (normal, not huge) for the pair fluxes: the hardware's approximate reciprocal
// (PTX rcp.approx.ftz.f64) refined by two Newton-Raphson steps for f(y) = 1/y - x,
// y <- y + y (1 - x y), each computed with fused multiply-adds.  The approximation's relative error
// is squared by every step, so two steps reach double precision (within an ulp of the rounded
// quotient); the denominators here are products of densities, inverse temperatures and their log
// means, far from zero and from overflow.  It replaces the longer IEEE division sequence (one per pair).
__device__ __forceinline__ double rcp_nr(double x) {
  double y;
  asm("rcp.approx.ftz.f64 %0, %1;" : "=d"(y) : "d"(x));
  double e = fma(-x, y, 1.0);
  y = fma(y, e, y);
  e = fma(-x, y, 1.0);
  return fma(y, e, y);
}

// log mean of (a, b) as num/den given la = log(a), lb = log(b)
__device__ __forceinline__ void ln_mean_nd(double a, double b, double la, double lb, double& num, double& den) {
  const double d = b - a, s = b + a;
  const double d2 = d * d, s2 = s * s;
  const double qs = s2 * (s2 * (s2 + d2 * (1. / 3.)) + d2 * d2 * (1. / 5.)) + d2 * d2 * d2 * (1. / 7.);
  const bool series = d2 < 1.0e-4 * s2;
  num = series ? 0.5 * s * (s2 * s2 * s2) : d;
  den = series ? qs : (lb - la);
}

// log mean of (a, b) = (L[i], R[i]) as num/den; the logarithms log a = L[il], log b = R[il] are read
// only off the series branch (R usually points into shared memory: in smooth flows nearly every
// pair takes the series branch, so its two logarithm loads are skipped)
__device__ __forceinline__ void ln_mean_nd(const double* L, const double* R, int i, int il, double& num,
                                           double& den) {
  const double a = L[i], b = R[i];
  const double d = b - a, s = b + a;
  const double d2 = d * d, s2 = s * s;
  if (d2 < 1.0e-4 * s2) {
    num = 0.5 * s * (s2 * s2 * s2);
    den = s2 * (s2 * (s2 + d2 * (1. / 3.)) + d2 * d2 * (1. / 5.)) + d2 * d2 * d2 * (1. / 7.);
  } else {
    num = d;
    den = R[il] - L[il];
  }
}

// Record of a node in shared memory: NQ flux quantities at [0, NQ), the metric terms Ja^1..Ja^3
// (x,y,z each) at [MO, MO+9), RS doubles per node.  The odd stride RS spreads the records of the
// nodes of a line over the shared-memory banks (padded 16-byte-aligned records read with 16-byte
// loads measured 19 % slower on the N=7 volume kernel).
template <int VF>
struct VolRec;
// standard DG (0) and dealiased metric (1): rho, rho u, rho v, rho w, rho E, u, v, w, p
template <> struct VolRec<0> { static constexpr int NQ = 9, MO = 9, RS = 19; };
template <> struct VolRec<1> { static constexpr int NQ = 9, MO = 9, RS = 19; };
// Kennedy-Gruber (2): rho, u, v, w, p, e = E/rho
template <> struct VolRec<2> { static constexpr int NQ = 6, MO = 6, RS = 15; };
// Ducros (3): halves of rho, u, v, w, p, rho u, rho v, rho w, rho E (every average is arithmetic)
template <> struct VolRec<3> { static constexpr int NQ = 9, MO = 9, RS = 19; };
// Morinishi (4): rho, u, v, w, p, |v|^2
template <> struct VolRec<4> { static constexpr int NQ = 6, MO = 6, RS = 15; };
// EC-KEP (5): rho, u/2, v/2, w/2, beta = rho/(2p), |v|^2/2, log rho, log beta (the halves make the
// pair averages plain sums; halving is exact, so the averages are bit-identical)
template <> struct VolRec<5> { static constexpr int NQ = 8, MO = 8, RS = 17; };
// approximate EC-KEP (6): rho/2, u/2, v/2, w/2, beta, |v|^2/2
template <> struct VolRec<6> { static constexpr int NQ = 6, MO = 6, RS = 15; };
// EC-KEP with pressure average (7): rho/2, u/2, v/2, w/2, p/2, beta, |v|^2/2, log beta
template <> struct VolRec<7> { static constexpr int NQ = 8, MO = 8, RS = 17; };
// Kennedy-Gruber, Pirozzoli form (8): halves of rho, u, v, w, p, H = (rho E + p)/rho
template <> struct VolRec<8> { static constexpr int NQ = 6, MO = 6, RS = 15; };
// Gassner-Winters-Walch (9): halves of sqrt(rho) times (1, u, v, w, H)
template <> struct VolRec<9> { static constexpr int NQ = 5, MO = 5, RS = 15; };
// Ismail-Roe (10): z1 = sqrt(rho/p), u, v, w, z5 = z1 p, log z1, log z5
template <> struct VolRec<10> { static constexpr int NQ = 7, MO = 7, RS = 17; };
// Ranocha (32): rho, u, v, w, p, rho/p, log rho, log(rho/p)
template <> struct VolRec<32> { static constexpr int NQ = 8, MO = 8, RS = 17; };

// the NQ flux quantities of record r (shared memory)
template <int VF>
__device__ __forceinline__ void load_rec(const double* r, double* q) {
#pragma unroll
  for (int z = 0; z < VolRec<VF>::NQ; ++z) q[z] = r[z];
}

// the metric triple Ja^(dir+1) of record r
template <int VF>
__device__ __forceinline__ void load_metric(const double* r, int dir, double* m) {
  const int off = VolRec<VF>::MO + 3 * dir;
  m[0] = r[off]; m[1] = r[off + 1]; m[2] = r[off + 2];
}

template <int VF>
__device__ __forceinline__ void make_record(const KParams& P, const double* U, double* r) {
  const double srho = 1. / U[0];
  const double u = U[1] * srho, v = U[2] * srho, w = U[3] * srho;
  const double v2 = u * u + v * v + w * w;
  const double p = P.kappaM1 * (U[4] - 0.5 * U[0] * v2);
  if constexpr (VF == 0 || VF == 1) {
    r[0] = U[0]; r[1] = U[1]; r[2] = U[2]; r[3] = U[3]; r[4] = U[4];
    r[5] = u; r[6] = v; r[7] = w; r[8] = p;
  } else if constexpr (VF == 2) {
    r[0] = U[0]; r[1] = u; r[2] = v; r[3] = w; r[4] = p; r[5] = srho * U[4];
  } else if constexpr (VF == 3) {
    r[0] = 0.5 * U[0]; r[1] = 0.5 * u; r[2] = 0.5 * v; r[3] = 0.5 * w; r[4] = 0.5 * p;
    r[5] = 0.5 * U[1]; r[6] = 0.5 * U[2]; r[7] = 0.5 * U[3]; r[8] = 0.5 * U[4];
  } else if constexpr (VF == 4) {
    r[0] = U[0]; r[1] = u; r[2] = v; r[3] = w; r[4] = p; r[5] = v2;
  } else if constexpr (VF == 6) {
    r[0] = 0.5 * U[0]; r[1] = 0.5 * u; r[2] = 0.5 * v; r[3] = 0.5 * w; r[4] = 0.5 * U[0] / p; r[5] = 0.5 * v2;
  } else if constexpr (VF == 7) {
    const double beta = 0.5 * U[0] / p;
    r[0] = 0.5 * U[0]; r[1] = 0.5 * u; r[2] = 0.5 * v; r[3] = 0.5 * w; r[4] = 0.5 * p; r[5] = beta;
    r[6] = 0.5 * v2; r[7] = log(beta);
  } else if constexpr (VF == 8) {
    r[0] = 0.5 * U[0]; r[1] = 0.5 * u; r[2] = 0.5 * v; r[3] = 0.5 * w; r[4] = 0.5 * p;
    r[5] = 0.5 * ((U[4] + p) * srho);
  } else if constexpr (VF == 9) {
    const double w1 = sqrt(U[0]);
    r[0] = 0.5 * w1; r[1] = 0.5 * (w1 * u); r[2] = 0.5 * (w1 * v); r[3] = 0.5 * (w1 * w);
    r[4] = 0.5 * (w1 * srho * (U[4] + p));
  } else if constexpr (VF == 5) {
    const double beta = 0.5 * U[0] / p;
    r[0] = U[0]; r[1] = 0.5 * u; r[2] = 0.5 * v; r[3] = 0.5 * w; r[4] = beta; r[5] = 0.5 * v2;
    r[6] = log(U[0]); r[7] = log(beta);
  } else if constexpr (VF == 10) {
    const double z1 = sqrt(U[0] / p);
    const double z5 = z1 * p;
    r[0] = z1; r[1] = u; r[2] = v; r[3] = w; r[4] = z5; r[5] = log(z1); r[6] = log(z5);
  } else if constexpr (VF == 32) {
    const double rsp = U[0] / p;
    r[0] = U[0]; r[1] = u; r[2] = v; r[3] = w; r[4] = p; r[5] = rsp; r[6] = log(U[0]); r[7] = log(rsp);
  }
}

// F = F#(L, R) . metric, symmetric in (L, R)
template <int VF>
__device__ __forceinline__ void pair_flux(const KParams& P, const double* L, const double* R, const double* mL,
                                          const double* mR, double* F) {
  if constexpr (VF == 0) {  // StandardDGFluxVec :394-439
    const double qL = L[5] * mL[0] + L[6] * mL[1] + L[7] * mL[2];
    const double qR = R[5] * mR[0] + R[6] * mR[1] + R[7] * mR[2];
    F[0] = 0.5 * (L[0] * qL + R[0] * qR);
    F[1] = 0.5 * (L[1] * qL + R[1] * qR + mL[0] * L[8] + mR[0] * R[8]);
    F[2] = 0.5 * (L[2] * qL + R[2] * qR + mL[1] * L[8] + mR[1] * R[8]);
    F[3] = 0.5 * (L[3] * qL + R[3] * qR + mL[2] * L[8] + mR[2] * R[8]);
    F[4] = 0.5 * ((L[4] + L[8]) * qL + (R[4] + R[8]) * qR);
  } else {
    // the records of these fluxes hold half metrics: the dealiased metric 1/2 (Ja_L + Ja_R) is a sum
    const double m1 = mL[0] + mR[0], m2 = mL[1] + mR[1], m3 = mL[2] + mR[2];
    if constexpr (VF == 1) {  // StandardDGFluxDealiasedMetricVec :446-494
      const double qL = L[5] * m1 + L[6] * m2 + L[7] * m3;
      const double qR = R[5] * m1 + R[6] * m2 + R[7] * m3;
      const double ps = L[8] + R[8];
      F[0] = 0.5 * (L[0] * qL + R[0] * qR);
      F[1] = 0.5 * (L[1] * qL + R[1] * qR + m1 * ps);
      F[2] = 0.5 * (L[2] * qL + R[2] * qR + m2 * ps);
      F[3] = 0.5 * (L[3] * qL + R[3] * qR + m3 * ps);
      F[4] = 0.5 * ((L[4] + L[8]) * qL + (R[4] + R[8]) * qR);
    } else if constexpr (VF == 2) {  // KennedyAndGruberFluxVec1 :731-803
      const double rhoHat = 0.5 * (L[0] + R[0]);
      const double uH = 0.5 * (L[1] + R[1]), vH = 0.5 * (L[2] + R[2]), wH = 0.5 * (L[3] + R[3]);
      const double p1 = 0.5 * (L[4] + R[4]);
      const double eH = 0.5 * (L[5] + R[5]);
      const double q = uH * m1 + vH * m2 + wH * m3;
      F[0] = rhoHat * q;
      F[1] = F[0] * uH + m1 * p1;
      F[2] = F[0] * vH + m2 * p1;
      F[3] = F[0] * wH + m3 * p1;
      F[4] = F[0] * eH + p1 * q;
    } else if constexpr (VF == 3) {  // DucrosFluxVec :986-1059 (records hold halves)
      const double q = (L[1] + R[1]) * m1 + (L[2] + R[2]) * m2 + (L[3] + R[3]) * m3;
      const double p1 = L[4] + R[4];
      F[0] = (L[0] + R[0]) * q;
      F[1] = (L[5] + R[5]) * q + m1 * p1;
      F[2] = (L[6] + R[6]) * q + m2 * p1;
      F[3] = (L[7] + R[7]) * q + m3 * p1;
      F[4] = ((L[8] + R[8]) + p1) * q;
    } else if constexpr (VF == 4) {  // MorinishiFluxVec :1121-1205
      const double uH = 0.5 * (L[1] + R[1]), vH = 0.5 * (L[2] + R[2]), wH = 0.5 * (L[3] + R[3]);
      const double p1 = 0.5 * (L[4] + R[4]);
      const double qL = L[1] * m1 + L[2] * m2 + L[3] * m3;
      const double qR = R[1] * m1 + R[2] * m2 + R[3] * m3;
      const double rq2L = 0.5 * L[0] * qL, rq2R = 0.5 * R[0] * qR;
      F[0] = rq2L + rq2R;
      F[1] = F[0] * uH + m1 * p1;
      F[2] = F[0] * vH + m2 * p1;
      F[3] = F[0] * wH + m3 * p1;
      F[4] = 0.5 * (P.kappa * P.sKappaM1 * (L[4] * qL + R[4] * qR) - (rq2L * L[5] + rq2R * R[5])) +
             rq2L * (L[1] * uH + L[2] * vH + L[3] * wH) + rq2R * (R[1] * uH + R[2] * vH + R[3] * wH);
    } else if constexpr (VF == 6) {  // EntropyAndEnergyConservingFluxVec2 :1427-1504 (halves)
      const double rhoM = L[0] + R[0];
      const double sbM = 2. * rcp_nr(L[4] + R[4]);
      const double uH = L[1] + R[1], vH = L[2] + R[2], wH = L[3] + R[3];
      const double p1 = 0.5 * rhoM * sbM;
      const double q = uH * m1 + vH * m2 + wH * m3;
      F[0] = rhoM * q;
      F[1] = F[0] * uH + m1 * p1;
      F[2] = F[0] * vH + m2 * p1;
      F[3] = F[0] * wH + m3 * p1;
      F[4] = F[0] * 0.5 * (P.sKappaM1 * sbM - (L[5] + R[5])) + uH * F[1] + vH * F[2] + wH * F[3];
    } else if constexpr (VF == 7) {  // ggFluxVec :1575-1653 (halves)
      double nb, db;
      ln_mean_nd(L, R, 5, 7, nb, db);
      const double rhoM = L[0] + R[0];
      const double uH = L[1] + R[1], vH = L[2] + R[2], wH = L[3] + R[3];
      const double p1 = L[4] + R[4];
      const double q = uH * m1 + vH * m2 + wH * m3;
      F[0] = rhoM * q;
      F[1] = F[0] * uH + m1 * p1;
      F[2] = F[0] * vH + m2 * p1;
      F[3] = F[0] * wH + m3 * p1;
      F[4] = F[0] * 0.5 * (P.sKappaM1 * (db * rcp_nr(nb)) - (L[6] + R[6])) + uH * F[1] + vH * F[2] + wH * F[3];
    } else if constexpr (VF == 8) {  // KennedyAndGruberFluxVec2 :857-929 (halves)
      const double uH = L[1] + R[1], vH = L[2] + R[2], wH = L[3] + R[3];
      const double p1 = L[4] + R[4];
      const double q = uH * m1 + vH * m2 + wH * m3;
      F[0] = (L[0] + R[0]) * q;
      F[1] = F[0] * uH + m1 * p1;
      F[2] = F[0] * vH + m2 * p1;
      F[3] = F[0] * wH + m3 * p1;
      F[4] = F[0] * (L[5] + R[5]);
    } else if constexpr (VF == 9) {  // GassnerWintersWalchFluxVec :1724-1799 (halves)
      const double rhoH = L[0] + R[0];
      const double uH = L[1] + R[1], vH = L[2] + R[2], wH = L[3] + R[3];
      const double HH = L[4] + R[4];
      const double p1 = P.kappaM1 * P.sKappa * (rhoH * HH - 0.5 * (uH * uH + vH * vH + wH * wH));
      const double q = uH * m1 + vH * m2 + wH * m3;
      F[0] = rhoH * q;
      F[1] = q * uH + m1 * p1;
      F[2] = q * vH + m2 * p1;
      F[3] = q * wH + m3 * p1;
      F[4] = q * HH;
    } else if constexpr (VF == 5) {  // EntropyAndEnergyConservingFluxVec :1277-1356
      double nr, dr, nb, db;
      ln_mean_nd(L, R, 0, 6, nr, dr);
      ln_mean_nd(L, R, 4, 7, nb, db);
      const double sr = L[0] + R[0], sb = L[4] + R[4];
      const double inv = rcp_nr(dr * sb * nb);
      const double rhoHat = nr * sb * nb * inv;      // LN(rho)
      const double p1 = 0.5 * sr * dr * nb * inv;    // 0.5*rho_mean/beta_mean
      const double sbHat = db * dr * sb * inv;       // 1/LN(beta)
      const double uH = L[1] + R[1], vH = L[2] + R[2], wH = L[3] + R[3];  // records hold u/2, v/2, w/2
      const double q = uH * m1 + vH * m2 + wH * m3;
      F[0] = rhoHat * q;
      F[1] = F[0] * uH + m1 * p1;
      F[2] = F[0] * vH + m2 * p1;
      F[3] = F[0] * wH + m3 * p1;
      F[4] = F[0] * 0.5 * (P.sKappaM1 * sbHat - (L[5] + R[5])) + uH * F[1] + vH * F[2] + wH * F[3];
    } else if constexpr (VF == 10) {  // TwoPointEntropyConservingFluxVec :574-673
      double n1, d1, n5, d5;
      ln_mean_nd(L, R, 0, 5, n1, d1);
      ln_mean_nd(L, R, 4, 6, n5, d5);
      const double z1M = 0.5 * (L[0] + R[0]);
      const double inv = rcp_nr(d5 * z1M * n1);
      const double z5LN = n5 * z1M * n1 * inv;
      const double sz1M = d5 * n1 * inv;
      const double ratio = n5 * d1 * z1M * inv;  // z5LN / z1LN
      const double rhoHat = z1M * z5LN;
      const double uH = 0.5 * (L[0] * L[1] + R[0] * R[1]) * sz1M;
      const double vH = 0.5 * (L[0] * L[2] + R[0] * R[2]) * sz1M;
      const double wH = 0.5 * (L[0] * L[3] + R[0] * R[3]) * sz1M;
      const double p1 = 0.5 * (L[4] + R[4]) * sz1M;
      const double q = uH * m1 + vH * m2 + wH * m3;
      F[0] = rhoHat * q;
      F[1] = F[0] * uH + m1 * p1;
      F[2] = F[0] * vH + m2 * p1;
      F[3] = F[0] * wH + m3 * p1;
      F[4] = 0.5 * (q * P.kappaP1 * P.sKappaM1 * ratio + uH * F[1] + vH * F[2] + wH * F[3]);
    } else if constexpr (VF == 32) {  // RanochaFluxVec :1876-1929
      double nr, dr, ns, ds;
      ln_mean_nd(L, R, 0, 6, nr, dr);
      ln_mean_nd(L, R, 5, 7, ns, ds);
      const double inv = rcp_nr(dr * ns);
      const double rhoLN = nr * ns * inv;
      const double srspM = ds * dr * inv;  // 1/LN(rho/p)
      const double va1 = 0.5 * (L[1] + R[1]), va2 = 0.5 * (L[2] + R[2]), va3 = 0.5 * (L[3] + R[3]);
      const double v2zip = 0.5 * (L[1] * R[1] + L[2] * R[2] + L[3] * R[3]);
      const double pavg = 0.5 * (L[4] + R[4]);
      const double vmL = L[1] * m1 + L[2] * m2 + L[3] * m3;
      const double vmR = R[1] * m1 + R[2] * m2 + R[3] * m3;
      F[0] = rhoLN * 0.5 * (vmL + vmR);
      F[1] = F[0] * va1 + m1 * pavg;
      F[2] = F[0] * va2 + m2 * pavg;
      F[3] = F[0] * va3 + m3 * pavg;
      F[4] = F[0] * (v2zip + srspM * P.sKappaM1) + 0.5 * (L[4] * vmR + R[4] * vmL);
    }
  }
}

}  // namespace fluxo
