"""Benchmark of the reference's headline metric on the B200 path.

Workload (the configuration the reference's PID metric is quoted on here): compressible
Navier-Stokes Taylor-Green vortex, FP64, N=7, 32^3 hexahedra on [-pi,pi]^3 with interior nodes
deformed by 0.05*sin(x)sin(y)sin(z) (NGeo=2, curved metrics), Re=1600 (mu0=1/1600), Ma=0.1,
Pr=0.72, BR1 lifting of the entropy variables, EC-KEP split-form volume flux (VolumeFlux=5),
entropy-stable matrix-dissipation surface flux (Riemann=44), Carpenter LSERK4-5, CFLscale 0.5, DFLscale 0.5
(the reference's own TGV setup, ini/navstokes/tgv/parameter.ini; at CFLscale 0.9 the scheme is unstable
on this case: a 1e-14 perturbation of the initial state grows to 1e-2 in 60 steps).
Synthetic data: the mesh and the initial state are generated in-code (no mesh file, no dataset).

One step = CALCTIMESTEP + one 5-stage LSERK step (5 right-hand sides).  The metric is the
reference's PID per RHS evaluation, ns per DOF per RHS (lower is better); `value` is the whole-job
figure: timed seconds / (total DOFs over all ranks * RHS evaluations).  The state (671 MB) is
larger than L2, so no extra flush is needed between steps.

Multi-GPU: independent replicas, one per rank (weak scaling); the timed region is bracketed by a
barrier + device synchronisation and the maximum over ranks is reported.
"""
import argparse
import json
import os
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

# Algorithmic FP64 operations per DOF of one right-hand side for this workload, from one RHS of
# the CPU oracle's counting build (oracle/counted.h rules), split by the phase that each GPU
# kernel implements.  tests/test_bench_constants.py re-derives these numbers.
FALG_PER_DOF = {
    "volume_split_form": 1124.5,
    "lifting": 519.75,
    "volume_viscous": 384.0,
    "face_flux": 200.625,
    "surface_integral": 7.5,
    "jacobian_source": 5.0,
}
FALG_RK_STAGE_PER_DOF = 20.0  # Ut_tmp = Ut - A*Ut_tmp; U += b*dt*Ut_tmp (2+2 flops x 5 variables)
# Work of each kernel of one right-hand side (the phases it computes).  The viscous volume integral
# (volint.f90:228-271) is computed by the lifting kernel, which hands the volume kernel its result.
VOLUME_KERNEL_FALG = (FALG_PER_DOF["volume_split_form"] + FALG_PER_DOF["surface_integral"] +
                      FALG_PER_DOF["jacobian_source"] + FALG_RK_STAGE_PER_DOF)
LIFTING_KERNEL_FALG = FALG_PER_DOF["lifting"] + FALG_PER_DOF["volume_viscous"]
# Compulsory bytes per face point of the HBM-bound face kernels (face points per DOF: 3/(N+1)):
#   face_flux: U traces of both sides (2 x 5), n, t1, t2, SurfElem (10), n.F_v traces (2 x 4) read,
#              the flux (5) written = 33 doubles;
#   lift_flux: U traces of both sides (10) and SurfElem (1) read, the lifting flux (5) written = 16.
FACE_FLUX_BYTES_PER_POINT = 33 * 8
LIFT_FLUX_BYTES_PER_POINT = 16 * 8

# ncu figures of the shipped kernels.  DRAM bytes (read + write) per DOF of one launch of this
# workload at its full size (32^3, one-pass capture of one time step's stages >= 2,
# profiles/launches_dram_ns_tgv_N7_32x32x32.md); the FP64 pipe's active fraction
# (sm__pipe_fp64_cycles_active, --set full on the 16^3 case, profiles/*_ns_tgv_N7_16x16x16.md), which
# the F_alg fraction sits below where a kernel spends FP64 instructions that F_alg counts as one flop
# (division, logarithm) or issues products and sums that a multiply-add would fuse.
NCU_DRAM_BYTES_PER_DOF = {"volume": 321.0, "gradient": 209.1, "face_flux": 107.9, "lift_flux": 47.8}
NCU_FP64_PIPE_ACTIVE = {"volume": 0.458, "gradient": 0.204, "face_flux": 0.372}  # gradient: DMMA tiles 0.119 more
VOLUME_KERNEL_DRAM_BYTES_PER_DOF = NCU_DRAM_BYTES_PER_DOF["volume"]

METRIC = "PID ns/DOF/RHS, NS Taylor-Green N=7 32^3 curved, BR1 + EC-KEP + ES (Riemann 44), LSERK4-5"

# The resistive-MHD configuration (--workload mhd): F_alg per DOF of one RHS by phase, from the
# oracle's counting build on the configuration's initial state (4^3 elements, N=4); the NFVSE
# phase is zero there because the smooth initial data blends no element.
MHD_FALG_PER_DOF = {
    "volume_split_form": 1912.0,
    "lifting": 787.6,
    "volume_viscous": 510.0,
    "face_flux": 850.692,
    "surface_integral": 21.6,
    "jacobian_source": 9.0,
}
MHD_VOLUME_KERNEL_FALG = (MHD_FALG_PER_DOF["volume_split_form"] + MHD_FALG_PER_DOF["surface_integral"] +
                          MHD_FALG_PER_DOF["jacobian_source"] + 36.0)  # + LSERK stage, 4 flops x 9 variables
MHD_METRIC = ("PID ns/DOF/RHS, resistive MHD+GLM Orszag-Tang N=4 24^3 curved, Derigs EC + 9-wave ES "
              "(Riemann 14), Powell, BR1, NFVSE, LSERK4-5")


# The batched configuration (--workload batch): F_alg per DOF of one RHS for each (equation, N) of the
# mix (EC-KEP volume flux + Riemann 44 for both; Navier-Stokes with BR1), from the oracle's counting
# build on a 2^3 instance with the mix's initial data (fourier_state, seed SEED).
BATCH_FALG_PER_DOF = {
    (0, 3): 783.5859375, (0, 4): 877.212, (0, 5): 992.2013888888889, (0, 7): 1249.1220703125,
    (1, 3): 1632.5859375, (1, 4): 1738.812, (1, 5): 1882.201388888889, (1, 7): 2219.6220703125,
}
BATCH_METRIC = ("aggregate DOF-updates/s (DOFs x RHS evaluations per second), 64 uneven Euler/NS periodic-box "
                "instances (4^3..16^3 elements, N in {3,4,5,7}) batched, vs one at a time")
SERVE_METRIC = ("served DOF-updates/s with p50/p99 time-to-solution, Poisson stream of Euler/NS periodic-box "
                "solves (4^3..24^3 elements, N 3..7, end time log-uniform [0.05,1]), continuous batching vs one "
                "at a time")


def mhd_workload(elems=24, N=4):
    return dict(N=N, elems=(elems,) * 3, xmin=(0.0,) * 3, xmax=(2 * np.pi,) * 3, NGeo=2, deform_amp=0.05,
                eqn=3, lifting=1, lifting_var=3, riemann=14, volume_flux=10, kappa=5.0 / 3.0, eta=1e-3, mu0=0.0,
                noncons=1, nc_glm=0, glm_scale=0.5, nfvse=1, compute_alpha=1, alpha_max=0.5, alpha_min=0.01,
                space_prop_sweeps=1, cfl_scale=0.5, dfl_scale=0.5, time_disc=0)  # as ini/mhd/orszagtang


def workload(elems=32, N=7):
    return dict(N=N, elems=(elems,) * 3, xmin=(-np.pi,) * 3, xmax=(np.pi,) * 3, NGeo=2, deform_amp=0.05,
                eqn=1, lifting=1, lifting_var=3, visc=0, riemann=44, volume_flux=5, mu0=1.0 / 1600.0, Pr=0.72,
                kappa=1.4, ini_exact_func=7, cfl_scale=0.5, dfl_scale=0.5, time_disc=0)


def config_dict(w, n_gpus, steps):
    return {"workload": "navierstokes_tgv_N%d_%dx%dx%d_curved" % ((w["N"],) + w["elems"]), "N": w["N"],
            "elements": list(w["elems"]), "dofs_per_gpu": int(np.prod(w["elems"]) * (w["N"] + 1) ** 3),
            "riemann": w["riemann"], "volume_flux": w["volume_flux"], "lifting": "br1_entropy_var",
            "time_disc": "carpenterrk4-5", "rhs_per_step": 5, "parallelism": "replicas x%d" % n_gpus,
            "l2": "inputs larger than L2 (state 671 MB)", "steps": steps}


# ------------------------------------------------------------------------------------------------
class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled every 100 ms; the summary keeps the samples whose
    timestamps fall in the timed region (the sampler is started, and its first sample awaited, before
    the region begins; when the region is shorter than the period the nearest sample stands in)."""

    Q = ("timestamp,index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.f = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
        self.p = None
        self.t0 = self.t1 = None

    def __enter__(self):
        try:
            self.p = subprocess.Popen(["nvidia-smi", "-i", str(self.index), "--query-gpu=" + self.Q,
                                       "--format=csv,noheader,nounits", "-lms", "100"], stdout=self.f,
                                      stderr=subprocess.DEVNULL)
            deadline = time.time() + 3.0
            while time.time() < deadline and os.path.getsize(self.f.name) == 0:
                time.sleep(0.02)
        except OSError:
            self.p = None
        self.t0 = time.time()
        return self

    def __exit__(self, *a):
        self.t1 = time.time()
        if self.p is not None:
            time.sleep(0.15)  # one more sample after the region
            self.p.terminate()
            try:
                self.p.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.p.kill()

    def summary(self):
        import datetime

        self.f.flush()
        self.f.seek(0)
        rows = []
        for line in self.f.read().strip().splitlines():
            r = [x.strip() for x in line.split(",")]
            try:
                ts = datetime.datetime.strptime(r[0], "%Y/%m/%d %H:%M:%S.%f").timestamp()
                rows.append((ts, r))
            except (ValueError, IndexError):
                continue
        os.unlink(self.f.name)
        inside = [r for ts, r in rows if self.t0 is not None and self.t0 <= ts <= self.t1]
        if not inside and rows and self.t0 is not None:
            mid = 0.5 * (self.t0 + self.t1)
            inside = [min(rows, key=lambda x: abs(x[0] - mid))[1]]
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for r in inside:
            try:
                sm.append(float(r[2]))
                mx = float(r[3])
                for k, nm in enumerate(names):
                    if r[6 + k].lower() == "active":
                        reasons.add(nm)
            except (ValueError, IndexError):
                continue
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm), "timed_s": (self.t1 - self.t0) if self.t0 is not None else None}


def dist_setup(n_gpus):
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import datetime

        import torch.distributed as dist

        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))
    return world, rank, local


def max_over_ranks(x, world, device):
    if world == 1:
        return x
    import torch
    import torch.distributed as dist

    t = torch.tensor([x], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def barrier(world):
    if world > 1:
        import torch.distributed as dist

        dist.barrier()


# ------------------------------------------------------------------------------------------------
def cpu_baseline(threads, seconds=15.0):
    """The oracle (a C++ restatement of the reference loop by loop, OpenMP over elements) timed on
    the host cores on a bounded sample of the same workload: 4^3 elements of the N=7 TGV."""
    os.environ["OMP_NUM_THREADS"] = str(threads)
    from oracle.oracle import OracleCase

    w = workload(elems=4)
    c = OracleCase(N=w["N"], nElems=w["elems"], xmin=w["xmin"], xmax=w["xmax"], NGeo=w["NGeo"],
                   deform_amp=w["deform_amp"], eqn=1, lifting=1, lifting_var=3, mu0=w["mu0"], riemann=44,
                   volume_flux=5, ini_exact_func=7, cfl_scale=w["cfl_scale"],
                   dfl_scale=w["dfl_scale"])
    U0 = c.get_U()
    t_sim, n = c.run(0.0, 1e9, max_iter=1)  # warm-up
    if n != 1:
        raise RuntimeError("oracle warm-up step failed: calc_timestep=%r" % (c.calc_timestep(),))
    nd = c.nElems * c.np ** 3
    t0 = time.perf_counter()
    steps = 0
    while time.perf_counter() - t0 < seconds:
        if steps % 50 == 0:  # restart from t=0: the coarse 4^3 sample is under-resolved for long runs
            c.set_U(U0)
            t_sim = 0.0
        t_sim, n = c.run(t_sim, 1e9, max_iter=1)
        if n != 1:
            raise RuntimeError("oracle step failed: calc_timestep=%r" % (c.calc_timestep(),))
        steps += n
    el = time.perf_counter() - t0
    pid = el / (nd * 5 * steps) * 1e9
    return {"value": pid, "unit": "ns/DOF/RHS", "cores": threads, "kind": "port",
            "sample": "oracle, TGV N=7 4x4x4 elements (32768 DOFs), %d LSERK4-5 steps in %.1f s" % (steps, el)}


def cpu_baseline_subprocess(threads, seconds):
    """cpu_baseline in a fresh interpreter, so the CPU run shares nothing with the GPU process."""
    env = dict(os.environ, OMP_NUM_THREADS=str(threads))
    code = ("import json, sys; sys.path.insert(0, %r); import bench; "
            "print(json.dumps(bench.cpu_baseline(%d, %r)))" % (ROOT, threads, float(seconds)))
    try:
        r = subprocess.run([sys.executable, "-c", code], env=env, capture_output=True, text=True,
                           timeout=seconds * 4 + 120)
        out = [x for x in r.stdout.splitlines() if x.startswith("{")]
        if r.returncode != 0 or not out:
            return {"error": (r.stderr or r.stdout)[-400:]}
        return json.loads(out[-1])
    except subprocess.TimeoutExpired:
        return {"error": "cpu baseline timed out"}


def run_reference(args):
    world, rank, _ = dist_setup(args.gpus)
    if rank != 0:
        return
    threads = os.cpu_count() or 1
    steps = []
    for _ in range(args.warmup):
        cpu_baseline(threads, seconds=1.0)
    for _ in range(args.steps):
        steps.append(cpu_baseline(threads, seconds=max(2.0, 60.0 / max(args.steps, 1))))
    vals = [s["value"] for s in steps]
    v = float(np.median(vals))
    w = workload()
    line = {"impl": "reference", "metric": METRIC, "value": v, "unit": "ns/DOF/RHS", "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": None, "higher_is_better": False,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": config_dict(w, args.gpus, args.steps),
            "cpu_baseline": dict(steps[-1], value=v),
            "e2e": {"value": v, "unit": "ns/DOF/RHS", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
            "note": "reference Fortran not buildable here (no Fortran compiler/MPI/HDF5); its C++ restatement "
                    "(oracle) runs on %d host threads" % threads}
    print(json.dumps(line))


def run_fluxo(args):
    import torch

    import fluxo_b200 as fb
    from fluxo_b200.solver import fp64_peak, get_state_ptr, profile, set_profiling, set_state_ptr

    world, rank, local = dist_setup(args.gpus)
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    mhd = args.workload == "mhd"
    t0 = time.time()
    if mhd:
        from fluxo_b200.workloads import mhd_orszag_tang_state

        w = mhd_workload(elems=args.elems or 24, N=args.N or 4)
        if args.shock_blend > 0:  # fixed blending (ComputeAlpha 3) so that the subcell kernel does work
            w.update(compute_alpha=3, shock_blend_coef=args.shock_blend)
        w.update(sub_fv_method=args.sub_fv, recons_boundaries=3 if args.sub_fv > 1 else 1,
                 nfvse_corr=1 if args.nfvse_corr else 0)
        nt = 1 if args.nodes == "gauss" else 2
        if nt == 1:  # the NFVSE subcells need LGL nodes: the Gauss variant runs the pure DG scheme
            w.update(nfvse=0, nfvse_corr=0, node_type=1)
        mesh = fb.box_mesh(w["N"], w["elems"], w["xmin"], w["xmax"], NGeo=w["NGeo"], deform_amp=w["deform_amp"],
                           node_type=nt)
        fields = {k: v for k, v in w.items() if k not in ("elems", "xmin", "xmax", "NGeo", "deform_amp")}
        U0 = mhd_orszag_tang_state(mesh["Elem_xGP"], kappa=w["kappa"])
        if args.shard and world > 1 and nt == 2:  # one solve over the ranks (set_partition is collective)
            from fluxo_b200.shard import DistExchange, ShardedOperator

            shard = ShardedOperator(mesh, world, rank, DistExchange, device=local, **fields)
            op = shard.op
            U0 = shard.part.local_state(U0)
            nd_total = int(np.prod(w["elems"])) * (w["N"] + 1) ** 3
        else:
            op = fb.DGOperator(device=local, **fields)
            op.set_mesh(mesh)
    else:
        w = workload(elems=args.elems or 32, N=args.N or 7)
        nt = 1 if args.nodes == "gauss" else 2
        mesh = fb.box_mesh(w["N"], w["elems"], w["xmin"], w["xmax"], NGeo=w["NGeo"], deform_amp=w["deform_amp"],
                           node_type=nt)
        tgv_fields = dict(N=w["N"], eqn=1, riemann=w["riemann"], volume_flux=w["volume_flux"], lifting=1,
                          lifting_var=3, visc=0, mu0=w["mu0"], Pr=w["Pr"], kappa=w["kappa"],
                          cfl_scale=w["cfl_scale"], dfl_scale=w["dfl_scale"], time_disc=0, node_type=nt)
        U0 = fb.exact_func(7, 0.0, mesh["Elem_xGP"], kappa=w["kappa"])
        if args.shard and world > 1:  # one solve over the ranks: owned elements + ghosts, NCCL exchanges
            from fluxo_b200.shard import DistExchange, ShardedOperator

            shard = ShardedOperator(mesh, world, rank, DistExchange, device=local, **tgv_fields)
            op = shard.op
            U0 = shard.part.local_state(U0)
            nd_total = int(np.prod(w["elems"])) * (w["N"] + 1) ** 3
        else:
            op = fb.DGOperator(device=local, **tgv_fields)
            op.set_mesh(mesh)
    del mesh
    op.set_state(U0)
    setup_s = time.time() - t0
    nvar = 9 if mhd else 5
    sharded = args.shard and world > 1 and args.nodes == "lgl"
    nd = (shard.part.n_owned if sharded else op.nElems) * (w["N"] + 1) ** 3
    if sharded:
        args.no_e2e, args.no_mix, args.no_cpu = True, True, True
    _, _, stream_ptr = op.device_buffers()
    stream = torch.cuda.ExternalStream(stream_ptr, device=dev)
    peak = fp64_peak(local)

    t = 0.0
    t, n, err = op.time_disc(t, 1e30, args.warmup)
    assert err == 0 and n == args.warmup

    # ---- device-resident timed region ----
    n0 = op.launch_count()
    set_profiling(op, True)
    barrier(world)
    torch.cuda.synchronize(dev)
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with ClockSampler(local) as clk:
        ev0.record(stream)
        t, n, err = op.time_disc(t, 1e30, args.steps)
        ev1.record(stream)
        torch.cuda.synchronize(dev)
    barrier(world)
    assert err == 0 and n == args.steps, (err, n)
    ms = ev0.elapsed_time(ev1)
    launches = op.launch_count() - n0
    vol_ms, vol_n = profile(op, 3)
    kinds = {k: profile(op, i)
             for i, k in enumerate(("lift_flux", "gradient", "face_flux", "volume", "timestep", "nfvse"))
             if i != 3 and (i != 5 or mhd)}
    kinds["volume"] = (vol_ms, vol_n)
    set_profiling(op, False)
    ms_max = max_over_ranks(ms, world, dev)
    rhs = 5 * args.steps
    value = ms_max * 1e6 / ((nd_total if sharded else world * nd) * rhs)

    # ---- end-to-end through the public API with pinned host buffers ----
    e2e = None
    if not args.no_e2e:
        hostU = torch.empty(nd * nvar, dtype=torch.float64, pin_memory=True)
        get_state_ptr(op, hostU.data_ptr())
        e2e_steps = max(2, min(args.steps, 5))
        barrier(world)
        torch.cuda.synchronize(dev)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(e2e_steps):
            set_state_ptr(op, hostU.data_ptr())
            t, n, err = op.time_disc(t, 1e30, 1)
            get_state_ptr(op, hostU.data_ptr())
        e1.record(stream)
        torch.cuda.synchronize(dev)
        barrier(world)
        ems = max_over_ranks(e0.elapsed_time(e1), world, dev)
        e2e = {"value": ems * 1e6 / (world * nd * 5 * e2e_steps), "unit": "ns/DOF/RHS",
               "h2d_bytes_per_step": nd * nvar * 8, "d2h_bytes_per_step": nd * nvar * 8, "steps": e2e_steps,
               "path": "fluxo_gpu_set_state + fluxo_gpu_time_disc(1 step) + fluxo_gpu_get_state, pinned host"}

    if rank != 0:
        op.close()
        return
    vol_avg_ms = vol_ms / max(vol_n, 1)
    vol_falg = MHD_VOLUME_KERNEL_FALG if mhd else VOLUME_KERNEL_FALG
    achieved = vol_falg * nd / (vol_avg_ms * 1e-3) / 1e12
    roofline = {"bound": "fp64", "kernel": "mhd::volume_kernel<5,10>" if mhd else "volume_kernel<8,5,true>",
                "achieved": achieved, "peak": peak, "unit": "TFLOP/s", "frac": achieved / peak,
                "traffic": None if mhd else VOLUME_KERNEL_DRAM_BYTES_PER_DOF * nd,
                "traffic_note": None if mhd else "DRAM bytes per launch, one-pass ncu capture of this workload",
                "flops_per_dof_launch": vol_falg, "launch_ms": vol_avg_ms,
                "fp64_pipe_active_ncu": None if mhd else NCU_FP64_PIPE_ACTIVE["volume"],
                "peak_source": "measured in this job: DFMA loop (fluxo_gpu_fp64_peak); MEASURED_PEAKS.json has no FP64"}
    gauss = args.nodes == "gauss"
    # Gauss nodes: the face pass also holds the prolongation and the surface kernel, so the per-kernel and
    # whole-RHS fractions (F_alg of the LGL scheme) do not apply
    per_kernel = None if (mhd or gauss or sharded) else kernel_rooflines(kinds, w["N"], nd, op.nElems, peak)
    falg_rhs = sum((MHD_FALG_PER_DOF if mhd else FALG_PER_DOF).values())
    if mhd:
        alpha = op.alpha()[: nd // (w["N"] + 1) ** 3] if w["nfvse"] else np.zeros(op.nElems)
        config = {"workload": "mhd_glm_resistive_orszag_tang_N%d_%dx%dx%d_curved" % ((w["N"],) + w["elems"]) +
                  ("_gauss_nodes_no_nfvse" if gauss else "") +
                  ("" if args.shock_blend <= 0 else "_blend%g" % args.shock_blend) +
                  ("" if args.sub_fv == 1 else "_subfv%d" % args.sub_fv) + ("_corr" if args.nfvse_corr else ""),
                  "N": w["N"], "elements": list(w["elems"]), "dofs_per_gpu": nd, "riemann": 14, "volume_flux": 10,
                  "noncons": "powell", "lifting": "br1_entropy_var", "eta": w["eta"],
                  "nfvse": "off (Gauss nodes)" if gauss else (
                      ("indicator, alpha_max 0.5, alpha_min 0.01, 1 sweep" if args.shock_blend <= 0 else
                       "fixed alpha %g (ComputeAlpha 3)" % args.shock_blend) +
                      ", SubFVMethod %d" % args.sub_fv + (", NFVSE_CORR" if args.nfvse_corr else "")),
                  "blended_elements_last_rhs": int((alpha > 0).sum()), "time_disc": "carpenterrk4-5",
                  "rhs_per_step": 5,
                  "parallelism": ("one solve over %d GPUs (contiguous element ranges + ghost elements, NCCL)" % world
                                  if sharded else "replicas x%d" % world),
                  "l2": "inputs larger than L2 (state %d MB)" % (nd * 72 // 10 ** 6), "steps": args.steps}
    else:
        config = config_dict(w, world, args.steps)
        if sharded:
            config["parallelism"] = "one solve over %d GPUs (contiguous element ranges + ghost elements, NCCL)" % world
            config["dofs_per_gpu"] = nd
        if gauss:
            config["workload"] += "_gauss_nodes"
            config["nodes"] = "Gauss (entropy-projected face states, FluxB surface correction)"
    line = {"metric": MHD_METRIC if mhd else METRIC, "value": value, "unit": "ns/DOF/RHS", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_max / args.steps,
            "higher_is_better": False, "scaling": "strong" if sharded else "weak", "vs_baseline": None,
            "dtype": "f64", "data": "synthetic",
            "config": config, "roofline": roofline, "roofline_kernels": per_kernel, "e2e": e2e,
            "gpu_launches": int(launches), "clocks": clk.summary(),
            "kernel_ms_per_step": {k: v[0] / args.steps for k, v in kinds.items()},
            "rhs_roofline_frac": None if gauss else (falg_rhs * nd * rhs / (ms * 1e-3) / 1e12) / peak,
            "setup_s": setup_s}
    if not mhd:
        line["volume_shape"] = shape_dict(w["N"], w["volume_flux"], True)
    if world == 1 and not args.no_cpu and not mhd:
        line["cpu_baseline"] = cpu_baseline_subprocess(os.cpu_count() or 1, seconds=args.cpu_seconds)
    op.close()
    if world == 1 and not mhd and not gauss and not args.no_mix:
        # the other half of the headline metric: batched vs plain and served p50/p99, on this GPU
        line["batch"] = measure_batch(args, world, rank, local, steps=args.mix_steps)
        line["serve"] = measure_serve(args, world, rank, local)
    print(json.dumps(line))


def hbm_peak():
    """Measured HBM copy bandwidth of this pool's B200s (MEASURED_PEAKS.json), else the fallback."""
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            return float(json.load(f)["hbm_gbs"]), "MEASURED_PEAKS.json hbm_gbs"
    except (OSError, KeyError, ValueError):
        return 6650.0, "fallback 6.65 TB/s"


def kernel_rooflines(kinds, N, nd, nElems, fp64_peak):
    """Per-kernel roofline of the Navier-Stokes right-hand side from the CUDA-event launch times:
    F_alg / time against the FP64 peak for the element kernels, compulsory bytes / time against the
    HBM copy bandwidth for the face kernels."""
    bw, bw_src = hbm_peak()
    npts = 3 * nElems * (N + 1) ** 2
    out = {}
    for k, name, falg in (("volume", "volume_kernel<%d,5,true>" % (N + 1), VOLUME_KERNEL_FALG),
                          ("gradient", "lift_visc_mma_kernel<1,3>" if N == 7 else "lift_visc_kernel<%d,1,3>" % (N + 1),
                           LIFTING_KERNEL_FALG)):
        ms, n = kinds.get(k, (0.0, 0))
        if n:
            a = falg * nd / (ms / n * 1e-3) / 1e12
            out[k] = {"kernel": name, "bound": "fp64", "launch_ms": ms / n, "flops_per_dof": falg, "achieved": a,
                      "peak": fp64_peak, "unit": "TFLOP/s", "frac": a / fp64_peak,
                      "fp64_pipe_active_ncu": NCU_FP64_PIPE_ACTIVE.get(k),
                      "dram_bytes_per_dof_ncu": NCU_DRAM_BYTES_PER_DOF.get(k)}
    for k, name, bpp in (("face_flux", "face_flux_kernel<44,1>", FACE_FLUX_BYTES_PER_POINT),
                         ("lift_flux", "lift_flux_kernel", LIFT_FLUX_BYTES_PER_POINT)):
        ms, n = kinds.get(k, (0.0, 0))
        if n:
            a = bpp * npts / (ms / n * 1e-3) / 1e9
            out[k] = {"kernel": name, "bound": "hbm", "launch_ms": ms / n, "bytes_per_face_point": bpp,
                      "achieved": a, "peak": bw, "unit": "GB/s", "frac": a / bw, "peak_source": bw_src,
                      "dram_bytes_per_dof_ncu": NCU_DRAM_BYTES_PER_DOF.get(k)}
    return out


def shape_dict(N, volume_flux, visc):
    """The volume kernel's launch shape the autotuner chose (index -1: not tuned)."""
    from fluxo_b200.solver import volume_shape

    count, index, epb, lpw = volume_shape(N, volume_flux, visc)
    return {"candidates": count, "chosen": index, "elements_per_block": epb, "lines_per_warp": lpw}


def batch_falg(specs):
    """Algorithmic FP64 operations of one RHS plus its LSERK stage update, summed over instances."""
    return sum((BATCH_FALG_PER_DOF[(s["eqn"], s["N"])] + FALG_RK_STAGE_PER_DOF) * s["elems"] ** 3 * (s["N"] + 1) ** 3
               for s in specs)


def batch_launches_per_step(specs):
    """Kernels in one replay of the batch's step graph: per group reset, CALCTIMESTEP, dt, time update,
    and per stage face + volume (+ lifting flux + gradients for Navier-Stokes)."""
    groups = {(s["eqn"], s["N"]) for s in specs}
    return sum(4 + 5 * (4 if eqn == 1 else 2) for eqn, _ in groups)


def run_batch(args):
    """The batched configuration on its own JSON line."""
    import torch

    world, rank, local = dist_setup(args.gpus)
    torch.cuda.set_device(local)
    line = measure_batch(args, world, rank, local)
    if rank == 0:
        print(json.dumps(line))


def measure_batch(args, world, rank, local, steps=None):
    """The batched configuration: the instances advance together (fluxo_batch_run, one graph replay
    per step) and, for comparison, one at a time (fluxo_gpu_time_disc per instance).  Returns the
    JSON line (rank 0; None elsewhere)."""
    import torch

    import fluxo_b200 as fb
    from fluxo_b200.batch import Batch
    from fluxo_b200.solver import fp64_peak
    from fluxo_b200.workloads import batch_instance_specs, build_instance, instance_fields

    dev = torch.device("cuda", local)
    nsteps = steps or nsteps
    t0 = time.time()
    specs = batch_instance_specs(args.instances)
    cache, insts = {}, []
    for s in specs:
        mesh, U = build_instance(s, cache)
        insts.append((s, mesh, U, fb.make_cfg(device=local, **instance_fields(s))))
    dofs = [s["elems"] ** 3 * (s["N"] + 1) ** 3 for s in specs]
    nd = sum(dofs)
    setup_s = time.time() - t0
    peak = fp64_peak(local)

    # ---- batched: all instances in one batch, one graph replay per step ----
    b = Batch(device=local)
    ids = [b.add(mesh, U, 0.0, 1e30, cfg=cfg) for (s, mesh, U, cfg) in insts]
    b.run(args.warmup)
    stream = torch.cuda.ExternalStream(b.stream(), device=dev)
    barrier(world)
    torch.cuda.synchronize(dev)
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with ClockSampler(local) as clk:
        ev0.record(stream)
        b.run(nsteps)
        ev1.record(stream)
        torch.cuda.synchronize(dev)
    barrier(world)
    ms = ev0.elapsed_time(ev1)
    for iid in ids:
        _, n, done, err = b.status(iid)
        assert n == args.warmup + nsteps and not done and err == 0, (iid, n, done, err)
    ms_max = max_over_ranks(ms, world, dev)
    value = world * nd * 5 * nsteps / (ms_max * 1e-3)
    groups, placed, nbytes = b.info()

    # ---- end to end through the public API: host state in and out every step ----
    e2e = None
    if not args.no_e2e:
        host = [torch.empty(d * 5, dtype=torch.float64, pin_memory=True) for d in dofs]
        for iid, h in zip(ids, host):
            b.lib.fluxo_batch_get_state(b.b, iid, h.data_ptr())
        e2e_steps = max(2, min(nsteps, 5))
        barrier(world)
        torch.cuda.synchronize(dev)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(e2e_steps):
            for iid, h in zip(ids, host):
                b._check(b.lib.fluxo_batch_set_state(b.b, iid, h.data_ptr()))
            b.run(1)
            for iid, h in zip(ids, host):
                b._check(b.lib.fluxo_batch_get_state(b.b, iid, h.data_ptr()))
        e1.record(stream)
        torch.cuda.synchronize(dev)
        barrier(world)
        ems = max_over_ranks(e0.elapsed_time(e1), world, dev)
        e2e = {"value": world * nd * 5 * e2e_steps / (ems * 1e-3), "unit": "DOF-updates/s",
               "h2d_bytes_per_step": nd * 5 * 8, "d2h_bytes_per_step": nd * 5 * 8, "steps": e2e_steps,
               "path": "fluxo_batch_set_state (all instances) + fluxo_batch_run(1) + fluxo_batch_get_state, pinned host"}
    b.close()

    # ---- one at a time: each instance alone through fluxo_gpu_time_disc, device time summed ----
    seq_ms, inst_ms = 0.0, []
    if not args.no_sequential:
        for (s, mesh, U, cfg) in insts:
            op = fb.DGOperator(cfg=cfg)
            op.set_mesh(mesh)
            op.set_state(U)
            t, n, err = op.time_disc(0.0, 1e30, args.warmup)
            st = torch.cuda.ExternalStream(op.device_buffers()[2], device=dev)
            torch.cuda.synchronize(dev)
            a0, a1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a0.record(st)
            t, n, err = op.time_disc(t, 1e30, nsteps)
            a1.record(st)
            torch.cuda.synchronize(dev)
            assert err == 0 and n == nsteps
            inst_ms.append(a0.elapsed_time(a1))
            op.close()
        seq_ms = max_over_ranks(sum(inst_ms), world, dev)
    # where batching pays: the instances of at most 8^3 elements, batched on their own vs alone
    small = None
    if inst_ms:
        sel = [k for k, s in enumerate(specs) if s["elems"] <= 8]
        bs = Batch(device=local)
        for k in sel:
            s, mesh, U, cfg = insts[k]
            bs.add(mesh, U, 0.0, 1e30, cfg=cfg)
        bs.run(args.warmup)
        sst = torch.cuda.ExternalStream(bs.stream(), device=dev)
        torch.cuda.synchronize(dev)
        b0, b1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        b0.record(sst)
        bs.run(nsteps)
        b1.record(sst)
        torch.cuda.synchronize(dev)
        bs.close()
        nds = sum(dofs[k] for k in sel)
        alone = sum(inst_ms[k] for k in sel)
        small = {"instances": len(sel), "dofs": nds, "batched_ms_per_step": b0.elapsed_time(b1) / nsteps,
                 "one_at_a_time_ms_per_step": alone / nsteps,
                 "batched_over_one_at_a_time": alone / b0.elapsed_time(b1),
                 "note": "instances of at most 8^3 elements: too small to fill the GPU alone"}
    if rank != 0:
        return None
    achieved = batch_falg(specs) * 5 * nsteps / (ms * 1e-3) / 1e12
    seq = None
    if seq_ms > 0:
        seq = {"value": world * nd * 5 * nsteps / (seq_ms * 1e-3), "unit": "DOF-updates/s",
               "ms_per_step": seq_ms / nsteps, "path": "fluxo_gpu_time_disc per instance, one after another"}
    ne = [s["elems"] ** 3 for s in specs]
    config = {"workload": "batched_%d_uneven_euler_ns_instances" % len(specs), "instances": len(specs),
              "elements": "per instance %d..%d (%d total)" % (min(ne), max(ne), sum(ne)),
              "N": sorted({s["N"] for s in specs}), "navier_stokes_instances": sum(s["eqn"] for s in specs),
              "dofs_per_gpu": nd, "groups": groups, "device_bytes": nbytes, "time_disc": "carpenterrk4-5",
              "rhs_per_step": 5, "parallelism": "replicas x%d" % world,
              "l2": "inputs larger than L2 (state %d MB)" % (nd * 40 // 10 ** 6), "steps": nsteps}
    line = {"metric": BATCH_METRIC, "value": value, "unit": "DOF-updates/s", "n_gpus": world, "steps": nsteps,
            "warmup": args.warmup, "ms_per_step": ms_max / nsteps, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic", "config": config,
            "roofline": {"bound": "fp64", "kernel": "batched step (all groups, all kernels)", "achieved": achieved,
                         "peak": peak, "unit": "TFLOP/s", "frac": achieved / peak, "traffic": None},
            "one_at_a_time": seq, "batched_over_one_at_a_time": (value / seq["value"]) if seq else None,
            "small_instances": small,
            "e2e": e2e, "gpu_launches": batch_launches_per_step(specs) * nsteps, "clocks": clk.summary(),
            "setup_s": setup_s,
            "volume_shapes": {"%s_N%d" % ("ns" if eqn else "euler", N): shape_dict(N, 5, eqn == 1)
                              for eqn, N in sorted({(s["eqn"], s["N"]) for s in specs})}}
    return line


def run_serve(args):
    """The served configuration on its own JSON line."""
    import torch

    world, rank, local = dist_setup(args.gpus)
    torch.cuda.set_device(local)
    line = measure_serve(args, world, rank, local)
    if rank == 0:
        print(json.dumps(line))


def measure_serve(args, world, rank, local):
    """The served configuration: a Poisson stream of solve requests, continuous batching under an HBM
    budget (fluxo_b200.serve.Server) vs the plain path serving them one at a time, first come first
    served.  Both arms see the same requests at the same arrival times (wall clock from the start of
    the arm); time-to-solution = completion on the host - arrival.  The budget is smaller than the
    stream's total device bytes, so admission waits for memory (the line records how often)."""
    import torch

    import fluxo_b200 as fb
    from fluxo_b200.batch import Batch, instance_bytes
    from fluxo_b200.serve import Request, Server, serve_one_at_a_time
    from fluxo_b200.workloads import SEED, build_instance, instance_fields, serve_request_specs

    dev = torch.device("cuda", local)
    t0 = time.time()
    specs = serve_request_specs(args.rate, args.duration, seed=SEED + rank)
    cache, reqs = {}, []
    for s in specs:
        mesh, U = build_instance(s, cache)
        reqs.append(Request(rid=s["index"], cfg=fb.make_cfg(device=local, **instance_fields(s)), mesh=mesh, U=U,
                            t_end=s["t_end"], arrival=s["arrival"]))
    del cache
    setup_s = time.time() - t0
    budget = int(args.hbm_budget_gb * 1e9)

    # warm-up: a short stream of the first requests (library, context and graph paths), untimed
    warm = [Request(rid=r.rid, cfg=r.cfg, mesh=r.mesh, U=r.U, t_end=r.t_end * 0.05, arrival=0.0) for r in reqs[:3]]
    b = Batch(device=local)
    with Server(b, budget, instance_bytes) as warm_srv:
        warm_srv.serve(warm)
    b.close()
    serve_one_at_a_time(warm[:1], lambda cfg: fb.DGOperator(cfg=cfg))

    barrier(world)
    torch.cuda.synchronize(dev)
    b = Batch(device=local)
    srv = Server(b, budget, instance_bytes, steps_per_poll=args.poll_steps, device_loop=not args.host_poll)
    with ClockSampler(local) as clk:
        served = srv.serve(reqs)
        torch.cuda.synchronize(dev)
    srv.close()
    b.close()
    barrier(world)
    plain = None
    if not args.no_sequential:
        plain = serve_one_at_a_time(reqs, lambda cfg: fb.DGOperator(cfg=cfg))
        torch.cuda.synchronize(dev)
    barrier(world)
    s_sum = served.summary()
    work = served.dof_updates()
    wall = max_over_ranks(served.wall, world, dev)
    value = world * work / wall
    p_sum = plain.summary() if plain else None
    if plain:
        p_sum["dof_updates_per_s"] = world * plain.dof_updates() / max_over_ranks(plain.wall, world, dev)
    if rank != 0:
        return None
    assert s_sum["requests"] == len(reqs), (s_sum["requests"], len(reqs))
    failed = [(r.rid, r.err, r.steps, r.t) for r in served.results if r.err]
    if failed:  # CALCTIMESTEP stopped these solves (errType); the plain path must stop them alike
        print("stopped requests (rid, errType, steps, t):", failed, file=sys.stderr)
        print("their specs:", [specs[f[0]] for f in failed], file=sys.stderr)
    dofs = [r.dofs for r in reqs]
    total_bytes = sum(instance_bytes(r.cfg, r.mesh["ElemToSide"].shape[0], r.mesh["SideToElem"].shape[0]) for r in reqs)
    config = {"workload": "served_stream_poisson_%greq_per_s_%gs" % (args.rate, args.duration),
              "requests": len(reqs), "rate_per_s": args.rate, "duration_s": args.duration,
              "elements": "per direction 4..24", "N": "3..7", "t_end": "log-uniform [0.05, 1]",
              "dofs_per_request": "%d..%d" % (min(dofs), max(dofs)), "hbm_budget_bytes": budget,
              "stream_device_bytes": total_bytes, "budget_binds": bool(total_bytes > budget and
                                                                       s_sum["max_running"] < len(reqs)),
              "requests_waiting_for_memory": s_sum["waited_for_memory"],
              "max_running": s_sum["max_running"], "max_device_bytes": s_sum["max_device_bytes"],
              "graph_rebuilds": served.rebuilds,
              "loop": ("host-polled, %d steps per poll" % args.poll_steps) if args.host_poll
              else "device-resident (CUDA graph while-node)",
              "device_loops": served.loops, "loop_wakes": served.wakes,
              "host_loop_start_s": served.start_s, "host_harvest_s": served.harvest_s,
              "stopped_by_calctimestep": len(failed),
              "parallelism": "replicas x%d (own stream per rank)" % world}
    line = {"metric": SERVE_METRIC, "value": value, "unit": "DOF-updates/s", "n_gpus": world, "steps": len(reqs),
            "warmup": len(warm), "ms_per_step": None, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic", "config": config,
            "p50_s": s_sum["p50_s"], "p99_s": s_sum["p99_s"], "mean_s": s_sum["mean_s"], "wall_s": wall,
            "one_at_a_time": p_sum,
            "served_over_one_at_a_time": (value / p_sum["dof_updates_per_s"]) if p_sum else None,
            "e2e": {"value": value, "unit": "DOF-updates/s",
                    "h2d_bytes_per_step": int(np.mean([r.U.nbytes for r in reqs])),
                    "d2h_bytes_per_step": int(np.mean([r.U.nbytes for r in reqs])),
                    "note": "a step is one request: its mesh and state go to the device at admission, its "
                            "state comes back at completion, all inside the served wall time"},
            "clocks": clk.summary(), "setup_s": setup_s}
    return line


def run_tgv_trace(args):
    """The Taylor-Green configuration run to t=1 as the reference's TimeDisc runs it: time steps between
    analysis points every 0.05 (dt clipped to each), and at each point a right-hand side plus the
    device-side analysis (kinetic energy, enstrophy, entropy).  Reports the trace, the time to solution
    and the PID over the whole run (analysis included)."""
    import torch

    import fluxo_b200 as fb

    world, rank, local = dist_setup(args.gpus)
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    w = workload(elems=args.elems or 32, N=args.N or 7)
    mesh = fb.box_mesh(w["N"], w["elems"], w["xmin"], w["xmax"], NGeo=w["NGeo"], deform_amp=w["deform_amp"])
    op = fb.DGOperator(N=w["N"], eqn=1, riemann=w["riemann"], volume_flux=w["volume_flux"], lifting=1, lifting_var=3,
                       visc=0, mu0=w["mu0"], Pr=w["Pr"], kappa=w["kappa"], cfl_scale=w["cfl_scale"],
                       dfl_scale=w["dfl_scale"], time_disc=0, device=local)
    op.set_mesh(mesh)
    op.set_state(fb.exact_func(7, 0.0, mesh["Elem_xGP"], kappa=w["kappa"]))
    del mesh
    nd = op.nElems * (w["N"] + 1) ** 3
    _, _, stream_ptr = op.device_buffers()
    stream = torch.cuda.ExternalStream(stream_ptr, device=dev)
    op.dg_time_derivative(0.0)  # first use: the volume kernel's launch-shape tuning happens here
    barrier(world)
    torch.cuda.synchronize(dev)
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    t, steps, trace, k = 0.0, 0, [], 0
    w0 = time.time()
    with ClockSampler(local) as clk:
        ev0.record(stream)
        while True:
            a = op.analyze(t)
            trace.append({"t": t, "steps": steps, "ekin": a["ekin"], "enstrophy": a["enstrophy"],
                          "entropy": a["entropy"]})
            if t >= 1.0:
                break
            k += 1
            t, n, err = op.time_disc(t, min(0.05 * k, 1.0))
            assert err == 0
            steps += n
        ev1.record(stream)
        torch.cuda.synchronize(dev)
    wall = time.time() - w0
    ms = max_over_ranks(ev0.elapsed_time(ev1), world, dev)
    op.close()
    if rank != 0:
        return
    rhs = 5 * steps + len(trace)  # stage right-hand sides + one per analysis point
    line = {"metric": "Taylor-Green time to solution (t=1) with kinetic-energy / enstrophy trace every 0.05",
            "value": ms * 1e-3, "unit": "s", "n_gpus": world, "steps": steps, "warmup": 0,
            "higher_is_better": False, "scaling": "weak", "dtype": "f64", "data": "synthetic",
            "config": dict(config_dict(w, world, steps), workload="navierstokes_tgv_to_t1_N%d_%dx%dx%d_curved"
                           % ((w["N"],) + w["elems"])),
            "pid_ns_per_dof_rhs": ms * 1e6 / (world * nd * rhs), "wall_s": wall, "trace": trace,
            "clocks": clk.summary()}
    print(json.dumps(line))


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=40)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="fluxo", choices=("fluxo", "reference"))
    ap.add_argument("--workload", default="tgv", choices=("tgv", "mhd", "batch", "serve", "tgv_trace"),
                    help="tgv: the headline Navier-Stokes configuration; mhd: the resistive-MHD configuration; "
                         "batch: uneven Euler/NS instances batched vs one at a time; serve: Poisson request "
                         "stream, continuous batching vs one at a time; tgv_trace: the headline configuration "
                         "to t=1 with its kinetic-energy / enstrophy trace")
    ap.add_argument("--instances", type=int, default=64, help="batch: number of instances")
    ap.add_argument("--no-sequential", action="store_true", help="batch/serve: skip the one-at-a-time comparison")
    ap.add_argument("--rate", type=float, default=20.0, help="serve: requests per second")
    ap.add_argument("--duration", type=float, default=3.0, help="serve: seconds of arrivals")
    ap.add_argument("--hbm-budget-gb", type=float, default=8.0,
                    help="serve: device bytes for admitted requests (below the default stream's total, so it binds)")
    ap.add_argument("--no-mix", action="store_true",
                    help="tgv: skip the batched and served measurements that the default line carries")
    ap.add_argument("--mix-steps", type=int, default=10, help="tgv: timed steps of the embedded batched measurement")
    ap.add_argument("--poll-steps", type=int, default=2,
                    help="serve with --host-poll: time steps between admission rounds")
    ap.add_argument("--host-poll", action="store_true",
                    help="serve: the host-polled loop (fluxo_batch_run) instead of the device-resident loop")
    ap.add_argument("--elems", type=int, default=0, help="elements per direction (0: the configuration's)")
    ap.add_argument("--N", type=int, default=0, help="polynomial degree (0: the configuration's)")
    ap.add_argument("--shock-blend", type=float, default=0.0,
                    help="mhd: fixed blending coefficient (ComputeAlpha 3) instead of the indicator")
    ap.add_argument("--sub-fv", type=int, default=1, choices=(1, 2, 3, 4), help="mhd: SubFVMethod")
    ap.add_argument("--nfvse-corr", action="store_true", help="mhd: NFVSE_CORR positivity correction")
    ap.add_argument("--shard", action="store_true",
                    help="tgv / mhd with --gpus > 1: one solve over the GPUs (strong scaling) instead of replicas")
    ap.add_argument("--nodes", default="lgl", choices=("lgl", "gauss"),
                    help="Gauss-Lobatto (the headline) or Gauss nodes (PP_NodeType; mhd: without NFVSE)")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--cpu-seconds", type=float, default=15.0)
    args = ap.parse_args()
    if args.impl == "reference":
        run_reference(args)
    elif args.workload == "batch":
        run_batch(args)
    elif args.workload == "serve":
        run_serve(args)
    elif args.workload == "tgv_trace":
        run_tgv_trace(args)
    else:
        run_fluxo(args)
    if int(os.environ.get("WORLD_SIZE", "1")) > 1:
        import torch.distributed as dist

        dist.destroy_process_group()


if __name__ == "__main__":
    main()
