// Batched solves: many independent Euler / Navier-Stokes instances (different meshes, N, end
// times) advanced together on one GPU.  The reference runs one solve per program; this layer sits
// above its DGTimeDerivative / TimeDisc path and reuses the same kernels:
//   * instances with the same kernel configuration (equation, N, fluxes, lifting, constants,
//     LSERK scheme) form a group whose element and side arrays are the concatenation of its
//     instances' arrays (connectivity offset), so one launch per kernel covers the whole group;
//   * every instance keeps its own time, end time and time step: CALCTIMESTEP reduces into a
//     per-instance minimum, the LSERK update reads the element's instance dt, and a finished
//     instance gets dt = 0 until it is removed;
//   * one time step of all groups (CALCTIMESTEP, the stages, the per-instance bookkeeping) is
//     captured once as a CUDA graph and replayed; the graph is captured again after instances join or
//     leave, when a run needs it;
//   * the request loop of a server runs on the device: a second graph repeats that step inside a
//     conditional while-node until an instance finishes, the host raises a wake word in mapped pinned
//     memory (a request can be admitted), or a step limit is reached (fluxo_batch_loop_start).
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <climits>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <map>
#include <string>
#include <vector>

#include "../../include/fluxo_gpu.h"
#include "common.cuh"
#include "host_setup.h"
#include "host_copy.h"
#include "launch.h"

using namespace fluxo;

namespace {

// per-instance time-loop state (device), the batch form of TimeDisc's loop variables (timedisc.f90:274-359)
struct InstState {
  double t, tEnd, dt;
  int iter, maxIter, last, done, err;
};

__global__ void batch_reset_kernel(int first, int n, unsigned long long* bits, int* key) {
  const int i = first + blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= first + n) return;
  bits[i] = 0x7FF0000000000000ull;
  key[i] = INT_MAX;
}

// after CALCTIMESTEP: per instance error check and dt clipping to its end time (timedisc.f90:289-317)
__global__ void batch_finalize_kernel(int first, int n, InstState* s, const unsigned long long* bits,
                                      const int* key, double* instDt) {
  const int i = first + blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= first + n) return;
  InstState& S = s[i];
  double dt = 0.;
  if (!S.done) {
    if (key[i] != INT_MAX) {
      S.err = key[i] & 7;
      S.done = 1;
    } else {
      dt = __longlong_as_double((long long)bits[i]);
      S.last = 0;
      if (S.tEnd - S.t <= dt * (1. + 1.e-4)) { dt = S.tEnd - S.t; S.last = 1; }
    }
  }
  S.dt = dt;
  instDt[i] = dt;
}

// after the stages: t += dt, iteration count, termination (timedisc.f90:329-359)
__global__ void batch_advance_kernel(int first, int n, InstState* s) {
  const int i = first + blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= first + n) return;
  InstState& S = s[i];
  if (S.done) return;
  S.t = S.t + S.dt;
  S.iter += 1;
  if (S.last || (S.maxIter > 0 && S.iter >= S.maxIter)) S.done = 1;
}

// Last node of the device-resident loop's body (one per time step): counts the unfinished instances
// and ends the while-loop (condition 0) when fewer are running than at the loop's start, when the
// host raised the wake word, or after loop[1] steps.  loop = {steps done, step limit, running at the
// start, end reason, running now}.  The step limit bounds every loop, whatever the host does.
__global__ void batch_loop_cond_kernel(cudaGraphConditionalHandle h, const InstState* s, int nInst, int* loop,
                                       const volatile int* wake) {
  __shared__ int running;
  if (threadIdx.x == 0) running = 0;
  __syncthreads();
  int r = 0;
  for (int i = threadIdx.x; i < nInst; i += blockDim.x) r += s[i].done ? 0 : 1;
  if (r) atomicAdd(&running, r);
  __syncthreads();
  if (threadIdx.x != 0) return;
  const int steps = loop[0] + 1;
  loop[0] = steps;
  int why = 0;
  if (running < loop[2]) why = FLUXO_LOOP_FINISHED;
  else if (*wake != 0) why = FLUXO_LOOP_WOKEN;
  else if (steps >= loop[1]) why = FLUXO_LOOP_STEP_LIMIT;
  loop[3] = why;
  loop[4] = running;
  cudaGraphSetConditional(h, why == 0 ? 1u : 0u);
}

// host copies of a placed instance, freed after the GPU work that follows the placement is enqueued
// (returning a large request's 1 GB to the system takes time the GPU need not wait for)
struct Retired {
  std::vector<double> met, sJ, geo, U;
};

struct Instance {
  int id = 0;
  fluxo_cfg cfg{};
  int nElems = 0, nSides = 0;
  std::vector<int> s2e, e2s;                  // local 0-based connectivity (kept for re-offsetting)
  std::vector<double> met, sJ, geo, U;        // host data until the instance is placed on the device
  bool placed = false, removed = false;
  int group = -1, elemOff = 0, sideOff = 0, slot = -1;
  InstState st{};                             // host copy of the time-loop state
};

struct Group {
  fluxo_cfg key{};
  int N = 0, NP = 0;
  bool visc = false;
  int nStages = 0;
  double RKA[24]{}, RKb[24]{}, RKc[24]{}, CFLScale = 0., DFLScale = 0.;
  int nElems = 0, nSides = 0;
  std::vector<int> members;                   // instance ids in placement order
  int slot0 = 0;                              // members own instance slots slot0 .. slot0+members-1
  BasisTables* dBasis = nullptr;
  double *U = nullptr, *Ut = nullptr, *UtTmp = nullptr, *metrics = nullptr, *sJ = nullptr, *facegeo = nullptr;
  double *flux = nullptr, *lflux = nullptr, *gtrace = nullptr, *utvisc = nullptr;
  int *s2e = nullptr, *e2s = nullptr, *elemInst = nullptr;
};

// the kernel configuration that groups instances (ini_* and device do not matter to the kernels)
fluxo_cfg group_key(const fluxo_cfg& c) {
  fluxo_cfg k;
  std::memset(&k, 0, sizeof(k));
  k.struct_size = c.struct_size; k.N = c.N; k.eqn = c.eqn; k.riemann = c.riemann; k.volume_flux = c.volume_flux;
  if (c.eqn == FLUXO_EQN_NAVIERSTOKES) {
    k.lifting = c.lifting; k.lifting_var = c.lifting_var; k.visc = c.visc;
    k.Pr = c.Pr; k.mu0 = c.mu0; k.Ts = c.Ts; k.Tref = c.Tref; k.ExpoSuth = c.ExpoSuth; k.ExpoPow = c.ExpoPow;
    k.etaBR2 = c.etaBR2; k.R = c.R; k.dfl_scale = c.dfl_scale;
  }
  k.kappa = c.kappa; k.time_disc = c.time_disc; k.cfl_scale = c.cfl_scale;
  return k;
}

}  // namespace

struct fluxo_batch {
  int device = 0;
  cudaStream_t stream = nullptr;
  std::map<int, Instance> inst;
  std::vector<Group> groups;
  int nextId = 1;
  bool dirty = false;
  int nInst = 0;                               // instances with a device slot
  InstState* dState = nullptr;
  double* dInstDt = nullptr;
  unsigned long long* dDtBits = nullptr;
  int* dErrKey = nullptr;
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  std::vector<cudaStream_t> branch;            // one capture stream per group
  std::vector<cudaEvent_t> joins;              // fork / join points of the capture
  // device-resident loop: the while-graph (captured at the first loop_start after a commit), the
  // mapped pinned words (wake word [0], loop words [8..12] copied in and out), the loop's end event
  cudaGraph_t loopGraph = nullptr;
  cudaGraphExec_t loopExec = nullptr;
  bool loopStale = true;
  int* hWords = nullptr;
  int* dWake = nullptr;
  int* dLoop = nullptr;
  InstState* hStates = nullptr;                // pinned copy of the states at the loop's end
  int hStatesCap = 0;
  cudaEvent_t loopEnd = nullptr;
  bool loopActive = false;
  std::vector<Retired> retired;                // host copies of newly placed instances (freed after launch)
  std::string lastError;
};

// an instance repacked on the host, not yet in a batch (fluxo_batch_prepare)
struct fluxo_batch_prepared {
  Instance inst;
};

namespace {

int bfail(fluxo_batch* b, int code, const std::string& msg) {
  if (b) b->lastError = msg;
  else record_unbound_error(code, msg);
  return code;
}

#define BATCH_CUDA(b, call)                                                                        \
  do {                                                                                             \
    cudaError_t _e = (call);                                                                       \
    if (_e != cudaSuccess) return bfail((b), FLUXO_ECUDA, std::string(#call) + ": " + cudaGetErrorString(_e)); \
  } while (0)

template <class T>
cudaError_t balloc(fluxo_batch* b, T** p, size_t n) {
  if (n == 0) n = 1;
  return cudaMallocAsync((void**)p, n * sizeof(T), b->stream);
}

// device bytes an instance occupies in its group's arrays (the sizes allocated in commit)
size_t instance_bytes(const fluxo_cfg& c, int ne, int ns) {
  const size_t NP = c.N + 1, NP3 = NP * NP * NP, NPT = NP * NP;
  size_t d = 3 * 5 * NP3 * ne + 9 * NP3 * ne + NP3 * ne + 10 * NPT * ns + 5 * NPT * ns;
  if (c.eqn == FLUXO_EQN_NAVIERSTOKES) d += 5 * NPT * ns + 4 * NP3 * ne + 8 * NPT * ns;
  return 8 * d + 4 * (5 * (size_t)ns + 12 * (size_t)ne + ne) + sizeof(InstState) + 8 + 8 + 4;
}

void free_group_arrays(fluxo_batch* b, Group& g) {
  void* ptrs[] = {g.U, g.Ut, g.UtTmp, g.metrics, g.sJ, g.facegeo, g.flux, g.lflux, g.gtrace, g.utvisc,
                  g.s2e, g.e2s, g.elemInst};
  for (void* p : ptrs)
    if (p) cudaFreeAsync(p, b->stream);
  g.U = g.Ut = g.UtTmp = g.metrics = g.sJ = g.facegeo = g.flux = g.lflux = g.gtrace = g.utvisc = nullptr;
  g.s2e = g.e2s = g.elemInst = nullptr;
}

KParams group_params(const fluxo_batch* b, const Group& g) {
  KParams P{};
  P.nElems = g.nElems; P.nSides = g.nSides;
  P.U = g.U; P.Ut = g.Ut; P.UtTmp = g.UtTmp; P.utvisc = g.utvisc;
  P.metrics = g.metrics; P.sJ = g.sJ; P.facegeo = g.facegeo;
  P.s2e = g.s2e; P.e2s = g.e2s;
  P.flux = g.flux; P.lflux = g.lflux; P.gtrace = g.gtrace;
  P.basis = g.dBasis;
  fill_ns_physics(P, g.key);
  P.CFLScale = g.CFLScale; P.DFLScale = g.DFLScale;
  // elemInst holds the instance's index within the group: the per-instance arrays start at slot0
  P.elemInst = g.elemInst;
  P.instDt = b->dInstDt + g.slot0; P.instDtBits = b->dDtBits + g.slot0; P.instErrKey = b->dErrKey + g.slot0;
  return P;
}

// One group's time step: CALCTIMESTEP into its instances' minima, dt of each instance, the LSERK
// stages, the per-instance time update.  Nothing here reads another group's data.
cudaError_t enqueue_group_step(const fluxo_batch* b, const Group& g, cudaStream_t s) {
  const int n = (int)g.members.size(), bs = 128, nb = (n + bs - 1) / bs;
  cudaError_t e;
  batch_reset_kernel<<<nb, bs, 0, s>>>(g.slot0, n, b->dDtBits, b->dErrKey);
  KParams P = group_params(b, g);
  if ((e = launch_timestep(g.NP, g.visc, g.nElems, s, P, b->dDtBits, b->dErrKey)) != cudaSuccess) return e;
  batch_finalize_kernel<<<nb, bs, 0, s>>>(g.slot0, n, b->dState, b->dDtBits, b->dErrKey, b->dInstDt);
  for (int st = 1; st <= g.nStages; ++st) {
    P.stage = st;
    P.rkA = g.RKA[st]; P.rkB = g.RKb[st]; P.rkC = g.RKc[st];
    if (g.visc) {
      if ((e = launch_lift_flux(g.NP, g.nSides, s, P)) != cudaSuccess) return e;
      if ((e = launch_gradient(g.NP, g.nElems, s, P)) != cudaSuccess) return e;
    }
    if ((e = launch_face_flux(g.key.riemann, g.visc, g.NP, g.nSides, s, P)) != cudaSuccess) return e;
    if ((e = launch_volume(g.NP, g.key.volume_flux, g.visc, g.nElems, s, P)) != cudaSuccess) return e;
  }
  batch_advance_kernel<<<nb, bs, 0, s>>>(g.slot0, n, b->dState);
  return cudaGetLastError();
}

// One time step of every group, captured from the batch stream: the groups are independent
// branches of the graph (forked from and joined back into the batch stream), so the small
// launches of different groups share the SMs.
cudaError_t enqueue_step(fluxo_batch* b) {
  cudaStream_t s = b->stream;
  cudaError_t e;
  std::vector<const Group*> live;
  for (const Group& g : b->groups)
    if (g.nElems > 0) live.push_back(&g);
  if (b->branch.size() < live.size() || b->joins.size() < live.size() + 1) return cudaErrorInvalidValue;
  cudaEvent_t fork = b->joins[live.size()];
  if ((e = cudaEventRecord(fork, s)) != cudaSuccess) return e;
  for (size_t k = 0; k < live.size(); ++k) {
    cudaStream_t bs = b->branch[k];
    if ((e = cudaStreamWaitEvent(bs, fork, 0)) != cudaSuccess) return e;
    if ((e = enqueue_group_step(b, *live[k], bs)) != cudaSuccess) return e;
    if ((e = cudaEventRecord(b->joins[k], bs)) != cudaSuccess) return e;
    if ((e = cudaStreamWaitEvent(s, b->joins[k], 0)) != cudaSuccess) return e;
  }
  return cudaGetLastError();
}

// Places new instances, drops removed ones, rebuilds the group arrays and the step graph.
int commit(fluxo_batch* b) {
  if (!b->dirty) return FLUXO_OK;
  cudaStream_t s = b->stream;
  BATCH_CUDA(b, cudaSetDevice(b->device));
  // host copies of the time-loop states of the placed instances
  if (b->nInst > 0) {
    std::vector<InstState> hs(b->nInst);
    BATCH_CUDA(b, cudaMemcpyAsync(hs.data(), b->dState, sizeof(InstState) * b->nInst, cudaMemcpyDeviceToHost, s));
    BATCH_CUDA(b, cudaStreamSynchronize(s));
    for (auto& kv : b->inst)
      if (kv.second.placed && kv.second.slot >= 0) kv.second.st = hs[kv.second.slot];
  }
  // new group layout: surviving placed members keep their order, new instances follow
  std::vector<Group> ng = b->groups;
  std::vector<char> changed(ng.size(), 0);
  for (size_t k = 0; k < ng.size(); ++k) {
    std::vector<int> keep;
    for (int id : ng[k].members)
      if (!b->inst[id].removed) keep.push_back(id);
    changed[k] = keep.size() != ng[k].members.size();
    ng[k].members = keep;
  }
  for (auto& kv : b->inst) {
    Instance& I = kv.second;
    if (I.placed || I.removed) continue;
    const fluxo_cfg key = group_key(I.cfg);
    int gi = -1;
    for (size_t k = 0; k < ng.size(); ++k)
      if (std::memcmp(&ng[k].key, &key, sizeof(key)) == 0) gi = (int)k;
    if (gi < 0) {
      Group g;
      g.key = key; g.N = I.cfg.N; g.NP = I.cfg.N + 1; g.visc = (I.cfg.eqn == FLUXO_EQN_NAVIERSTOKES);
      time_disc_setup(I.cfg, g.RKA, g.RKb, g.RKc, &g.nStages, &g.CFLScale, &g.DFLScale);
      BasisTables hb;
      basis_tables_for(g.N, hb);
      BATCH_CUDA(b, balloc(b, &g.dBasis, 1));
      BATCH_CUDA(b, cudaMemcpyAsync(g.dBasis, &hb, sizeof(hb), cudaMemcpyHostToDevice, s));
      BATCH_CUDA(b, cudaStreamSynchronize(s));  // hb is a stack copy
      ng.push_back(g);
      changed.push_back(1);
      gi = (int)ng.size() - 1;
    }
    ng[gi].members.push_back(I.id);
    changed[gi] = 1;
  }
  // dense instance slots in group order
  int slot = 0;
  std::vector<InstState> hs;
  for (Group& g : ng) {
    g.slot0 = slot;
    for (int id : g.members) {
      Instance& I = b->inst[id];
      I.slot = slot++;
      hs.push_back(I.st);
    }
  }
  const int nInst = slot;
  // allocate the new arrays of the groups whose membership changed and move / upload their data;
  // the other groups keep their arrays (their element -> instance map is group-local)
  for (size_t gi = 0; gi < ng.size(); ++gi) {
    if (!changed[gi]) continue;
    Group& g = ng[gi];
    const int NP = g.NP, NP3 = NP * NP * NP, NPT = NP * NP, NV = 5;
    int ne = 0, ns = 0;
    for (int id : g.members) { ne += b->inst[id].nElems; ns += b->inst[id].nSides; }
    Group old = (gi < b->groups.size()) ? b->groups[gi] : Group();
    g.nElems = ne; g.nSides = ns;
    g.U = g.Ut = g.UtTmp = g.metrics = g.sJ = g.facegeo = g.flux = g.lflux = g.gtrace = g.utvisc = nullptr;
    g.s2e = g.e2s = g.elemInst = nullptr;
    if (ne > 0) {
      const size_t nU = (size_t)NV * NP3 * ne;
      BATCH_CUDA(b, balloc(b, &g.U, nU));
      BATCH_CUDA(b, balloc(b, &g.Ut, nU));
      BATCH_CUDA(b, balloc(b, &g.UtTmp, nU));
      BATCH_CUDA(b, balloc(b, &g.metrics, (size_t)9 * NP3 * ne));
      BATCH_CUDA(b, balloc(b, &g.sJ, (size_t)NP3 * ne));
      BATCH_CUDA(b, balloc(b, &g.facegeo, (size_t)10 * NPT * ns));
      BATCH_CUDA(b, balloc(b, &g.flux, (size_t)5 * NPT * ns));
      BATCH_CUDA(b, balloc(b, &g.s2e, (size_t)5 * ns));
      BATCH_CUDA(b, balloc(b, &g.e2s, (size_t)12 * ne));
      BATCH_CUDA(b, balloc(b, &g.elemInst, (size_t)ne));
      if (g.visc) {
        BATCH_CUDA(b, balloc(b, &g.lflux, (size_t)5 * NPT * ns));
        BATCH_CUDA(b, balloc(b, &g.utvisc, (size_t)4 * NP3 * ne));
        BATCH_CUDA(b, balloc(b, &g.gtrace, (size_t)2 * 4 * NPT * ns));  // n.F_v of both sides
      }
      std::vector<int> s2e((size_t)5 * ns), e2s((size_t)12 * ne), einst(ne);
      int eo = 0, so = 0;
      for (int id : g.members) {
        Instance& I = b->inst[id];
        for (int sd = 0; sd < I.nSides; ++sd) {
          s2e[5 * (size_t)(so + sd) + 0] = I.s2e[5 * (size_t)sd + 0] + eo;
          s2e[5 * (size_t)(so + sd) + 1] = I.s2e[5 * (size_t)sd + 1] + eo;
          for (int c = 2; c < 5; ++c) s2e[5 * (size_t)(so + sd) + c] = I.s2e[5 * (size_t)sd + c];
        }
        for (int el = 0; el < I.nElems; ++el) {
          for (int ls = 0; ls < 6; ++ls) {
            e2s[12 * (size_t)(eo + el) + 2 * ls] = I.e2s[12 * (size_t)el + 2 * ls] + so;
            e2s[12 * (size_t)(eo + el) + 2 * ls + 1] = I.e2s[12 * (size_t)el + 2 * ls + 1];
          }
          einst[eo + el] = I.slot - g.slot0;
        }
        // element-sized data
        const size_t eU = (size_t)NV * NP3, eM = (size_t)9 * NP3, eJ = NP3, sG = (size_t)10 * NPT;
        if (I.placed) {
          BATCH_CUDA(b, cudaMemcpyAsync(g.U + eU * eo, old.U + eU * I.elemOff, eU * I.nElems * 8, cudaMemcpyDeviceToDevice, s));
          BATCH_CUDA(b, cudaMemcpyAsync(g.metrics + eM * eo, old.metrics + eM * I.elemOff, eM * I.nElems * 8,
                                        cudaMemcpyDeviceToDevice, s));
          BATCH_CUDA(b, cudaMemcpyAsync(g.sJ + eJ * eo, old.sJ + eJ * I.elemOff, eJ * I.nElems * 8, cudaMemcpyDeviceToDevice, s));
          BATCH_CUDA(b, cudaMemcpyAsync(g.facegeo + sG * so, old.facegeo + sG * I.sideOff, sG * I.nSides * 8,
                                        cudaMemcpyDeviceToDevice, s));
        } else {
          BATCH_CUDA(b, copy_h2d(g.U + eU * eo, I.U.data(), eU * I.nElems * 8, s));
          BATCH_CUDA(b, copy_h2d(g.metrics + eM * eo, I.met.data(), eM * I.nElems * 8, s));
          BATCH_CUDA(b, copy_h2d(g.sJ + eJ * eo, I.sJ.data(), eJ * I.nElems * 8, s));
          BATCH_CUDA(b, copy_h2d(g.facegeo + sG * so, I.geo.data(), sG * I.nSides * 8, s));
        }
        I.elemOff = eo; I.sideOff = so; I.group = (int)gi;
        eo += I.nElems; so += I.nSides;
      }
      BATCH_CUDA(b, cudaMemcpyAsync(g.s2e, s2e.data(), s2e.size() * 4, cudaMemcpyHostToDevice, s));
      BATCH_CUDA(b, cudaMemcpyAsync(g.e2s, e2s.data(), e2s.size() * 4, cudaMemcpyHostToDevice, s));
      BATCH_CUDA(b, cudaMemcpyAsync(g.elemInst, einst.data(), einst.size() * 4, cudaMemcpyHostToDevice, s));
      BATCH_CUDA(b, cudaMemsetAsync(g.Ut, 0, nU * 8, s));
      BATCH_CUDA(b, cudaMemsetAsync(g.UtTmp, 0, nU * 8, s));
      BATCH_CUDA(b, cudaStreamSynchronize(s));  // host vectors above go out of scope
    }
    if (gi < b->groups.size()) free_group_arrays(b, b->groups[gi]);
  }
  // instance states
  if (b->dState) { cudaFreeAsync(b->dState, s); cudaFreeAsync(b->dInstDt, s); cudaFreeAsync(b->dDtBits, s); cudaFreeAsync(b->dErrKey, s); }
  b->dState = nullptr; b->dInstDt = nullptr; b->dDtBits = nullptr; b->dErrKey = nullptr;
  BATCH_CUDA(b, balloc(b, &b->dState, (size_t)std::max(nInst, 1)));
  BATCH_CUDA(b, balloc(b, &b->dInstDt, (size_t)std::max(nInst, 1)));
  BATCH_CUDA(b, balloc(b, &b->dDtBits, (size_t)std::max(nInst, 1)));
  BATCH_CUDA(b, balloc(b, &b->dErrKey, (size_t)std::max(nInst, 1)));
  if (nInst > 0)
    BATCH_CUDA(b, cudaMemcpyAsync(b->dState, hs.data(), sizeof(InstState) * nInst, cudaMemcpyHostToDevice, s));
  BATCH_CUDA(b, cudaStreamSynchronize(s));
  // drop removed instances, free the host copies of the placed ones
  for (auto it = b->inst.begin(); it != b->inst.end();) {
    if (it->second.removed) { it = b->inst.erase(it); continue; }
    Instance& I = it->second;
    if (!I.placed) {
      I.placed = true;
      Retired r;
      r.met.swap(I.met); r.sJ.swap(I.sJ); r.geo.swap(I.geo); r.U.swap(I.U);
      b->retired.push_back(std::move(r));
    }
    ++it;
  }
  b->groups = ng;
  b->nInst = nInst;
  // the step graph
  if (b->exec) { cudaGraphExecDestroy(b->exec); b->exec = nullptr; }
  if (b->graph) { cudaGraphDestroy(b->graph); b->graph = nullptr; }
  if (b->loopExec) { cudaGraphExecDestroy(b->loopExec); b->loopExec = nullptr; }
  if (b->loopGraph) { cudaGraphDestroy(b->loopGraph); b->loopGraph = nullptr; }
  b->loopStale = true;
  while (b->branch.size() < b->groups.size()) {
    cudaStream_t st;
    BATCH_CUDA(b, cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
    b->branch.push_back(st);
  }
  while (b->joins.size() < b->groups.size() + 1) {
    cudaEvent_t ev;
    BATCH_CUDA(b, cudaEventCreateWithFlags(&ev, cudaEventDisableTiming));
    b->joins.push_back(ev);
  }
  // launch shapes of the volume kernels, tuned on the group's own arrays before the capture
  for (const Group& g : b->groups)
    if (g.nElems > 0 && volume_shape(g.NP, g.key.volume_flux, g.visc) < 0)
      BATCH_CUDA(b, tune_volume(g.NP, g.key.volume_flux, g.visc, g.nElems, s, group_params(b, g)));
  // the step graph itself is captured by the first fluxo_batch_run after this (a server that only
  // runs device-resident loops captures the loop graph alone)
  b->dirty = false;
  return FLUXO_OK;
}

// The step graph (one time step of all groups), captured when a run needs it.
int build_step_graph(fluxo_batch* b) {
  if (b->exec || b->nInst == 0) return FLUXO_OK;
  cudaStream_t s = b->stream;
  BATCH_CUDA(b, cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal));
  cudaError_t e = enqueue_step(b);
  cudaGraph_t gr = nullptr;
  cudaError_t e2 = cudaStreamEndCapture(s, &gr);
  if (e != cudaSuccess || e2 != cudaSuccess) {
    if (gr) cudaGraphDestroy(gr);
    return bfail(b, FLUXO_ECUDA, std::string("step capture: ") + cudaGetErrorString(e != cudaSuccess ? e : e2));
  }
  b->graph = gr;
  BATCH_CUDA(b, cudaGraphInstantiate(&b->exec, b->graph, 0));
  return FLUXO_OK;
}

// The device-resident loop graph: one conditional while-node whose body is the captured time step
// of all groups followed by batch_loop_cond_kernel.  Built after a commit, at the first loop_start.
int build_loop_graph(fluxo_batch* b) {
  if (!b->loopStale && b->loopExec) return FLUXO_OK;
  if (b->loopExec) { cudaGraphExecDestroy(b->loopExec); b->loopExec = nullptr; }
  if (b->loopGraph) { cudaGraphDestroy(b->loopGraph); b->loopGraph = nullptr; }
  cudaStream_t s = b->stream;
  cudaGraph_t lg = nullptr;
  BATCH_CUDA(b, cudaGraphCreate(&lg, 0));
  b->loopGraph = lg;
  cudaGraphConditionalHandle h;
  BATCH_CUDA(b, cudaGraphConditionalHandleCreate(&h, lg, 1u, cudaGraphCondAssignDefault));
  cudaGraphNodeParams np = {};
  np.type = cudaGraphNodeTypeConditional;
  np.conditional.handle = h;
  np.conditional.type = cudaGraphCondTypeWhile;
  np.conditional.size = 1;
  cudaGraphNode_t node;
  BATCH_CUDA(b, cudaGraphAddNode(&node, lg, nullptr, 0, &np));
  cudaGraph_t body = np.conditional.phGraph_out[0];
  BATCH_CUDA(b, cudaStreamBeginCaptureToGraph(s, body, nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal));
  cudaError_t e = enqueue_step(b);
  if (e == cudaSuccess) {
    batch_loop_cond_kernel<<<1, 256, 0, s>>>(h, b->dState, b->nInst, b->dLoop, b->dWake);
    e = cudaGetLastError();
  }
  cudaGraph_t out = nullptr;
  cudaError_t e2 = cudaStreamEndCapture(s, &out);
  if (e != cudaSuccess || e2 != cudaSuccess)
    return bfail(b, FLUXO_ECUDA, std::string("loop capture: ") + cudaGetErrorString(e != cudaSuccess ? e : e2));
  BATCH_CUDA(b, cudaGraphInstantiate(&b->loopExec, lg, 0));
  b->loopStale = false;
  return FLUXO_OK;
}

// pinned words, pinned state copy and the end event of the device-resident loop (first use)
int loop_resources(fluxo_batch* b) {
  if (!b->hWords) {
    BATCH_CUDA(b, cudaHostAlloc((void**)&b->hWords, 64 * sizeof(int), cudaHostAllocMapped));
    std::memset(b->hWords, 0, 64 * sizeof(int));
    BATCH_CUDA(b, cudaHostGetDevicePointer((void**)&b->dWake, b->hWords, 0));
    BATCH_CUDA(b, cudaMalloc((void**)&b->dLoop, 8 * sizeof(int)));
    BATCH_CUDA(b, cudaEventCreateWithFlags(&b->loopEnd, cudaEventDisableTiming));
  }
  if (b->hStatesCap < b->nInst) {
    if (b->hStates) cudaFreeHost(b->hStates);
    b->hStates = nullptr;
    b->hStatesCap = 0;
    BATCH_CUDA(b, cudaHostAlloc((void**)&b->hStates, sizeof(InstState) * (size_t)b->nInst, cudaHostAllocDefault));
    b->hStatesCap = b->nInst;
  }
  return FLUXO_OK;
}

// after the loop's end event: the instances' host states and the loop words
void loop_collect(fluxo_batch* b, int* steps, int* reason, int* nRunning) {
  const int* w = b->hWords + 8;
  for (auto& kv : b->inst)
    if (kv.second.placed && kv.second.slot >= 0 && kv.second.slot < b->nInst) kv.second.st = b->hStates[kv.second.slot];
  if (steps) *steps = w[0];
  if (reason) *reason = w[3];
  if (nRunning) *nRunning = w[4];
  b->loopActive = false;
}

#define BATCH_IDLE(b)                                                                              \
  do {                                                                                             \
    if ((b)->loopActive)                                                                           \
      return bfail((b), FLUXO_ENOTREADY, "a device-resident loop is running (loop_poll / loop_wait first)"); \
  } while (0)

int check_cfg(const fluxo_cfg* c, std::string& msg) {
  if (!c || c->struct_size != (int)sizeof(fluxo_cfg)) { msg = "fluxo_cfg size mismatch"; return FLUXO_EINVAL_CFG; }
  if (c->N < 1 || c->N > 7) { msg = "N must be in 1..7"; return FLUXO_EINVAL_CFG; }
  if (c->eqn != FLUXO_EQN_EULER && c->eqn != FLUXO_EQN_NAVIERSTOKES) {
    msg = "batched solves support the Euler and Navier-Stokes equations";
    return FLUXO_EINVAL_CFG;
  }
  if (!riemann_supported(c->riemann) || !volume_flux_supported(c->volume_flux)) {
    msg = "Riemann solver or volume flux not implemented";
    return FLUXO_EINVAL_CFG;
  }
  if (c->nfvse) {
    msg = "batched solves run without shock capturing";
    return FLUXO_EINVAL_CFG;
  }
  if (c->node_type == 1) {
    msg = "batched solves run on Gauss-Lobatto nodes";
    return FLUXO_EINVAL_CFG;
  }
  if (c->eqn == FLUXO_EQN_NAVIERSTOKES &&
      (c->lifting < 1 || c->lifting > 2 || c->lifting_var < 1 || c->lifting_var > 3 || c->visc < 0 || c->visc > 2)) {
    msg = "lifting / lifting_var / visc out of range";
    return FLUXO_EINVAL_CFG;
  }
  if (!(c->kappa > 1.)) { msg = "kappa must be > 1"; return FLUXO_EINVAL_CFG; }
  if (c->ini_exact_func == 4) { msg = "source terms are not supported in batches"; return FLUXO_EINVAL_CFG; }
  if (c->time_disc < 0 || c->time_disc > 5) {  // the fused stage update serves the LSERKW2 schemes 0..5
    msg = "batched solves take the two-register (LSERKW2) schemes, time_disc 0..5";
    return FLUXO_EINVAL_CFG;
  }
  return FLUXO_OK;
}

// Host-only part of an admission: configuration checks, the mesh repacked into the device layout,
// the initial state and time-loop state (no batch state is touched, so any host thread may run it).
int prepare_instance(const fluxo_cfg* cfg, int nElems, int nSides, const int* SideToElem, const int* ElemToSide,
                     const double* Mf, const double* Mg, const double* Mh, const double* sJ, const double* NormVec,
                     const double* TangVec1, const double* TangVec2, const double* SurfElem, const double* U,
                     double t, double tEnd, int maxIter, Instance& I, std::string& msg) {
  int r = check_cfg(cfg, msg);
  if (r) return r;
  if (nElems < 1 || nSides < 1 || !SideToElem || !ElemToSide || !Mf || !Mg || !Mh || !sJ || !NormVec || !TangVec1 ||
      !TangVec2 || !SurfElem || !U) {
    msg = "missing array";
    return FLUXO_EINVAL_CFG;
  }
  I.cfg = *cfg;
  I.nElems = nElems; I.nSides = nSides;
  if (!host::repack_mesh(cfg->N, nElems, nSides, SideToElem, ElemToSide, Mf, Mg, Mh, NormVec, TangVec1, TangVec2,
                         SurfElem, I.s2e, I.e2s, I.met, I.geo, msg))
    return FLUXO_EINVAL_CFG;
  const size_t NP3 = (size_t)(cfg->N + 1) * (cfg->N + 1) * (cfg->N + 1);
  I.sJ.assign(sJ, sJ + NP3 * nElems);
  I.U.assign(U, U + 5 * NP3 * nElems);
  I.st.t = t; I.st.tEnd = tEnd; I.st.dt = 0.; I.st.iter = 0; I.st.maxIter = maxIter; I.st.last = 0;
  I.st.done = (t >= tEnd || maxIter == 0) ? 1 : 0;
  I.st.err = 0;
  return FLUXO_OK;
}

void add_instance(fluxo_batch* b, Instance&& I, int* id) {
  I.id = b->nextId++;
  *id = I.id;
  b->inst[I.id] = std::move(I);
  b->dirty = true;
}

}  // namespace

extern "C" {

int fluxo_batch_create(int device, fluxo_batch** out) {
  if (!out) return bfail(nullptr, FLUXO_EINVAL_CFG, "null argument");
  *out = nullptr;
  fluxo_batch* b = new fluxo_batch();
  b->device = device;
  cudaError_t e = cudaSetDevice(device);
  if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking);
  if (e != cudaSuccess) {
    delete b;
    return bfail(nullptr, FLUXO_ECUDA, std::string("CUDA init: ") + cudaGetErrorString(e));
  }
  // keep freed blocks in the device's default pool, so rebuilding the groups re-uses them
  cudaMemPool_t pool;
  if (cudaDeviceGetDefaultMemPool(&pool, device) == cudaSuccess) {
    uint64_t thr = UINT64_MAX;
    cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &thr);
  }
  *out = b;
  return FLUXO_OK;
}

int fluxo_batch_prepare(const fluxo_cfg* cfg, int nElems, int nSides, const int* SideToElem, const int* ElemToSide,
                        const double* Mf, const double* Mg, const double* Mh, const double* sJ, const double* NormVec,
                        const double* TangVec1, const double* TangVec2, const double* SurfElem, const double* U,
                        double t, double tEnd, int maxIter, fluxo_batch_prepared** out) {
  if (!out) return bfail(nullptr, FLUXO_EINVAL_CFG, "batch_prepare: null argument");
  *out = nullptr;
  fluxo_batch_prepared* p = new fluxo_batch_prepared();
  std::string msg;
  const int r = prepare_instance(cfg, nElems, nSides, SideToElem, ElemToSide, Mf, Mg, Mh, sJ, NormVec, TangVec1,
                                 TangVec2, SurfElem, U, t, tEnd, maxIter, p->inst, msg);
  if (r) {
    delete p;
    return bfail(nullptr, r, "batch_prepare: " + msg);
  }
  *out = p;
  return FLUXO_OK;
}

int fluxo_batch_add_prepared(fluxo_batch* b, fluxo_batch_prepared* p, int* id) {
  if (!b || !p || !id) return bfail(b, FLUXO_EINVAL_CFG, "batch_add_prepared: null argument");
  add_instance(b, std::move(p->inst), id);
  delete p;
  return FLUXO_OK;
}

int fluxo_batch_prepared_free(fluxo_batch_prepared* p) {
  delete p;
  return FLUXO_OK;
}

int fluxo_batch_add(fluxo_batch* b, const fluxo_cfg* cfg, int nElems, int nSides, const int* SideToElem,
                    const int* ElemToSide, const double* Mf, const double* Mg, const double* Mh, const double* sJ,
                    const double* NormVec, const double* TangVec1, const double* TangVec2, const double* SurfElem,
                    const double* U, double t, double tEnd, int maxIter, int* id) {
  if (!b || !id) return bfail(b, FLUXO_EINVAL_CFG, "null argument");
  Instance I;
  std::string msg;
  const int r = prepare_instance(cfg, nElems, nSides, SideToElem, ElemToSide, Mf, Mg, Mh, sJ, NormVec, TangVec1,
                                 TangVec2, SurfElem, U, t, tEnd, maxIter, I, msg);
  if (r) return bfail(b, r, "batch_add: " + msg);
  add_instance(b, std::move(I), id);
  return FLUXO_OK;
}

int fluxo_batch_run(fluxo_batch* b, int nSteps, int* nRunning) {
  if (!b) return FLUXO_EINVAL_CFG;
  BATCH_IDLE(b);
  BATCH_CUDA(b, cudaSetDevice(b->device));
  int r = commit(b);
  if (r) return r;
  if ((r = build_step_graph(b))) return r;
  int running = 0;
  if (b->nInst > 0) {
    const int chunk = 8;
    std::vector<InstState> hs(b->nInst);
    for (int done = 0; done < nSteps;) {
      const int k = std::min(chunk, nSteps - done);
      for (int i = 0; i < k; ++i) BATCH_CUDA(b, cudaGraphLaunch(b->exec, b->stream));
      done += k;
      BATCH_CUDA(b, cudaMemcpyAsync(hs.data(), b->dState, sizeof(InstState) * b->nInst, cudaMemcpyDeviceToHost,
                                    b->stream));
      BATCH_CUDA(b, cudaStreamSynchronize(b->stream));
      running = 0;
      for (const InstState& S : hs) running += S.done ? 0 : 1;
      if (running == 0) break;
    }
    for (auto& kv : b->inst)
      if (kv.second.slot >= 0 && kv.second.slot < b->nInst) kv.second.st = hs[kv.second.slot];
  }
  b->retired.clear();
  if (nRunning) *nRunning = running;
  return FLUXO_OK;
}

int fluxo_batch_status(fluxo_batch* b, int id, double* t, int* nIter, int* done, int* errType) {
  if (!b) return FLUXO_EINVAL_CFG;
  auto it = b->inst.find(id);
  if (it == b->inst.end() || it->second.removed) return bfail(b, FLUXO_EINVAL_CFG, "unknown instance id");
  const InstState& S = it->second.st;
  if (t) *t = S.t;
  if (nIter) *nIter = S.iter;
  if (done) *done = S.done;
  if (errType) *errType = S.err;
  return FLUXO_OK;
}

int fluxo_batch_get_state(fluxo_batch* b, int id, double* U) {
  if (!b || !U) return FLUXO_EINVAL_CFG;
  BATCH_IDLE(b);
  auto it = b->inst.find(id);
  if (it == b->inst.end() || it->second.removed) return bfail(b, FLUXO_EINVAL_CFG, "unknown instance id");
  const Instance& I = it->second;
  const size_t n = (size_t)5 * (I.cfg.N + 1) * (I.cfg.N + 1) * (I.cfg.N + 1) * I.nElems;
  if (!I.placed) {
    std::copy(I.U.begin(), I.U.end(), U);
    return FLUXO_OK;
  }
  BATCH_CUDA(b, cudaSetDevice(b->device));
  const Group& g = b->groups[I.group];
  const size_t eU = (size_t)5 * g.NP * g.NP * g.NP;
  BATCH_CUDA(b, copy_d2h(U, g.U + eU * I.elemOff, n * 8, b->stream));
  return FLUXO_OK;
}

int fluxo_batch_set_state(fluxo_batch* b, int id, const double* U) {
  if (!b || !U) return FLUXO_EINVAL_CFG;
  BATCH_IDLE(b);
  auto it = b->inst.find(id);
  if (it == b->inst.end() || it->second.removed) return bfail(b, FLUXO_EINVAL_CFG, "unknown instance id");
  Instance& I = it->second;
  const size_t n = (size_t)5 * (I.cfg.N + 1) * (I.cfg.N + 1) * (I.cfg.N + 1) * I.nElems;
  if (!I.placed) {
    std::copy(U, U + n, I.U.begin());
    return FLUXO_OK;
  }
  BATCH_CUDA(b, cudaSetDevice(b->device));
  const Group& g = b->groups[I.group];
  const size_t eU = (size_t)5 * g.NP * g.NP * g.NP;
  BATCH_CUDA(b, copy_h2d(g.U + eU * I.elemOff, U, n * 8, b->stream));
  return FLUXO_OK;
}

int fluxo_batch_loop_start(fluxo_batch* b, int maxSteps) {
  if (!b || maxSteps < 1) return bfail(b, FLUXO_EINVAL_CFG, "loop_start: maxSteps must be >= 1");
  BATCH_IDLE(b);
  BATCH_CUDA(b, cudaSetDevice(b->device));
  int r = commit(b);
  if (r) return r;
  if ((r = loop_resources(b))) return r;
  int running = 0;
  for (const auto& kv : b->inst)
    if (kv.second.placed && !kv.second.removed && kv.second.slot >= 0 && !kv.second.st.done) ++running;
  int* w = b->hWords + 8;
  w[0] = 0; w[1] = maxSteps; w[2] = running; w[3] = FLUXO_LOOP_IDLE; w[4] = running;
  *(volatile int*)b->hWords = 0;  // wake word, lowered before the loop starts
  std::atomic_thread_fence(std::memory_order_seq_cst);
  if (running == 0 || b->nInst == 0) {  // nothing to advance: an empty loop that ends at once
    BATCH_CUDA(b, cudaEventRecord(b->loopEnd, b->stream));
    b->loopActive = true;
    for (int i = 0; i < b->nInst; ++i) b->hStates[i] = InstState{};
    for (const auto& kv : b->inst)
      if (kv.second.slot >= 0 && kv.second.slot < b->nInst) b->hStates[kv.second.slot] = kv.second.st;
    return FLUXO_OK;
  }
  if ((r = build_loop_graph(b))) return r;
  BATCH_CUDA(b, cudaMemcpyAsync(b->dLoop, w, 5 * sizeof(int), cudaMemcpyHostToDevice, b->stream));
  BATCH_CUDA(b, cudaGraphLaunch(b->loopExec, b->stream));
  BATCH_CUDA(b, cudaMemcpyAsync(w, b->dLoop, 5 * sizeof(int), cudaMemcpyDeviceToHost, b->stream));
  BATCH_CUDA(b, cudaMemcpyAsync(b->hStates, b->dState, sizeof(InstState) * b->nInst, cudaMemcpyDeviceToHost,
                                b->stream));
  BATCH_CUDA(b, cudaEventRecord(b->loopEnd, b->stream));
  b->loopActive = true;
  b->retired.clear();  // the uploads completed inside commit; freeing overlaps the loop
  return FLUXO_OK;
}

int fluxo_batch_loop_wake(fluxo_batch* b) {
  if (!b) return FLUXO_EINVAL_CFG;
  if (b->hWords) {
    *(volatile int*)b->hWords = 1;
    std::atomic_thread_fence(std::memory_order_seq_cst);
  }
  return FLUXO_OK;
}

int fluxo_batch_loop_poll(fluxo_batch* b, int* finished, int* steps, int* reason, int* nRunning) {
  if (!b || !finished) return FLUXO_EINVAL_CFG;
  *finished = 0;
  if (!b->loopActive) return bfail(b, FLUXO_ENOTREADY, "loop_poll: no loop was started");
  cudaError_t e = cudaEventQuery(b->loopEnd);
  if (e == cudaErrorNotReady) return FLUXO_OK;
  if (e != cudaSuccess) {
    b->loopActive = false;
    return bfail(b, FLUXO_ECUDA, std::string("loop_poll: ") + cudaGetErrorString(e));
  }
  loop_collect(b, steps, reason, nRunning);
  *finished = 1;
  return FLUXO_OK;
}

int fluxo_batch_loop_wait(fluxo_batch* b, int* steps, int* reason, int* nRunning) {
  if (!b) return FLUXO_EINVAL_CFG;
  if (!b->loopActive) return bfail(b, FLUXO_ENOTREADY, "loop_wait: no loop was started");
  cudaError_t e = cudaEventSynchronize(b->loopEnd);
  if (e != cudaSuccess) {
    b->loopActive = false;
    return bfail(b, FLUXO_ECUDA, std::string("loop_wait: ") + cudaGetErrorString(e));
  }
  loop_collect(b, steps, reason, nRunning);
  return FLUXO_OK;
}

int fluxo_batch_remove(fluxo_batch* b, int id) {
  if (!b) return FLUXO_EINVAL_CFG;
  auto it = b->inst.find(id);
  if (it == b->inst.end() || it->second.removed) return bfail(b, FLUXO_EINVAL_CFG, "unknown instance id");
  if (!it->second.placed) b->inst.erase(it);
  else it->second.removed = true;
  b->dirty = true;
  return FLUXO_OK;
}

int fluxo_batch_info(fluxo_batch* b, int* nGroups, int* nInstances, size_t* deviceBytes) {
  if (!b) return FLUXO_EINVAL_CFG;
  int ng = 0;
  for (const Group& g : b->groups) ng += g.nElems > 0 ? 1 : 0;
  if (nGroups) *nGroups = ng;
  if (nInstances) *nInstances = b->nInst;
  if (deviceBytes) {
    size_t d = 0;
    for (const auto& kv : b->inst)
      if (kv.second.placed && !kv.second.removed) d += instance_bytes(kv.second.cfg, kv.second.nElems, kv.second.nSides);
    *deviceBytes = d;
  }
  return FLUXO_OK;
}

int fluxo_batch_stream(fluxo_batch* b, void** stream) {
  if (!b || !stream) return FLUXO_EINVAL_CFG;
  *stream = (void*)b->stream;
  return FLUXO_OK;
}

int fluxo_batch_instance_bytes(const fluxo_cfg* cfg, int nElems, int nSides, size_t* bytes) {
  if (!cfg || !bytes || nElems < 0 || nSides < 0) return FLUXO_EINVAL_CFG;
  *bytes = instance_bytes(*cfg, nElems, nSides);
  return FLUXO_OK;
}

int fluxo_batch_last_error(fluxo_batch* b, char* buf, size_t len) {
  if (!b || !buf || len == 0) return FLUXO_EINVAL_CFG;
  std::snprintf(buf, len, "%s", b->lastError.c_str());
  return FLUXO_OK;
}

int fluxo_batch_destroy(fluxo_batch* b) {
  if (!b) return FLUXO_OK;
  cudaSetDevice(b->device);
  if (b->loopActive) fluxo_batch_loop_wake(b);  // a running loop ends after its current step
  if (b->stream) cudaStreamSynchronize(b->stream);
  if (b->exec) cudaGraphExecDestroy(b->exec);
  if (b->graph) cudaGraphDestroy(b->graph);
  if (b->loopExec) cudaGraphExecDestroy(b->loopExec);
  if (b->loopGraph) cudaGraphDestroy(b->loopGraph);
  if (b->hWords) cudaFreeHost(b->hWords);
  if (b->hStates) cudaFreeHost(b->hStates);
  if (b->dLoop) cudaFree(b->dLoop);
  if (b->loopEnd) cudaEventDestroy(b->loopEnd);
  for (Group& g : b->groups) {
    free_group_arrays(b, g);
    if (g.dBasis) cudaFreeAsync(g.dBasis, b->stream);
  }
  if (b->dState) { cudaFreeAsync(b->dState, b->stream); cudaFreeAsync(b->dInstDt, b->stream);
                   cudaFreeAsync(b->dDtBits, b->stream); cudaFreeAsync(b->dErrKey, b->stream); }
  if (b->stream) { cudaStreamSynchronize(b->stream); cudaStreamDestroy(b->stream); }
  for (cudaStream_t st : b->branch) cudaStreamDestroy(st);
  for (cudaEvent_t ev : b->joins) cudaEventDestroy(ev);
  delete b;
  return FLUXO_OK;
}

}  // extern "C"
