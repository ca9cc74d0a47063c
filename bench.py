"""Benchmark of the B200 solve path on the 'plain method at scale' workload.

Workload (one step = one pass of the hot path): the 64^3 hex grid of the unit
cube split into 6 tets per hex (1,572,864 TET4_EDGE elements), iron block
mu_r = 1000 in [0.25,0.75]^2 x [0.4,0.6], z-directed coil current on the
annulus 0.3 < r < 0.45, 0.2 < z < 0.8, n x A = 0 on all faces, reference tree
gauge (bit-exact numbering), FP64 assembly on the GPU (CSR pattern + K + F),
then Jacobi-PCG to a relative residual of 1e-8.  The edge numbering / gauge is
host integer setup done once per mesh (reported as setup_dof_ms).

`value` times the step with inputs resident in HBM (emg_system_create_typed on
device arrays + emg_system_assemble + emg_system_solve); `e2e` times the same C-ABI calls
with pinned host buffers (geometry and DOF map copied in, solution copied
out).
Both in solves/s; ms_per_step is the time to a 1e-8 residual.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl reference]
"""
from __future__ import annotations

import argparse
import ctypes as C
import gc
import json
import os
import statistics
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "time-to-1e-8 residual, learned+batched vs plain PCG/FETI-DP; SpMV GB/s vs HBM"
TOL = 1e-8
MAX_ITER = 50000


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--n", type=int, default=64, help="hex grid size (64 = the quoted workload)")
    ap.add_argument("--cpu-iters", type=int, default=250,
                    help="iterations in the CPU sample (about 10 s of 1-thread work at 64^3)")
    ap.add_argument("--no-cpu-baseline", action="store_true",
                    help="skip the CPU baseline (profiling runs)")
    ap.add_argument("--workload", default="cube64",
                    choices=["cube64", "hex64", "batch512", "fetidp64", "learned64"],
                    help="cube64: the plain method at scale (default line); batch512: 512 "
                         "independent 8^3..32^3 instances solved in one lockstep device loop; "
                         "fetidp64: the 64^3 problem split into 64 jittered box subdomains, "
                         "FETI-DP (factor + solve) next to plain PCG on the same gauged system; "
                         "hex64: the cube64 physics on 64^3 perturbed HEX8_EDGE elements")
    ap.add_argument("--parts", type=int, default=4, help="fetidp64: subdomains per axis")
    ap.add_argument("--train-fields", type=int, default=200, help="learned64: training fields (seeds 1000+)")
    ap.add_argument("--eval-fields", type=int, default=50, help="learned64: held-out fields (seeds 2000+)")
    ap.add_argument("--feti-precond", type=int, default=2,
                    help="fetidp64: 2 deluxe (FP64 blocks), 3 deluxe with FP32 blocks (mixed precision)")
    ap.add_argument("--cmp-train-fields", type=int, default=12,
                    help="cube64 metric comparison: training fields of the learned preconditioner")
    ap.add_argument("--cmp-eval-fields", type=int, default=3,
                    help="cube64 metric comparison: held-out fields of the learned preconditioner")
    ap.add_argument("--cmp-batch-instances", type=int, default=512,
                    help="cube64 metric comparison: instances of the batched many-instance run (0 skips it)")
    ap.add_argument("--feti-variants", default=",".join(["fp64", "fp32_precond", "tf32_factor"]),
                    help="cube64 metric comparison: FETI-DP variants to time (comma-separated)")
    ap.add_argument("--mixed", action="store_true",
                    help="fetidp64: mixed-precision factor (TF32 tensor-core contractions, FP64 refinement)")
    ap.add_argument("--instances", type=int, default=512, help="batch512: number of instances")
    ap.add_argument("--no-oracle", action="store_true",
                    help="cube64: skip the full-size FP64 oracle check after the timed region")
    ap.add_argument("--no-comparison", action="store_true",
                    help="cube64: skip the 64-subdomain FETI-DP comparison of the default line")
    ap.add_argument("--kernels-only", type=int, default=0, metavar="ITERS",
                    help="profiling mode: assemble once, then launch ITERS plain CG iterations "
                         "(no graphs) and print their per-kernel CUDA-event times")
    return ap.parse_args()


HEX_AMPLITUDE = 0.2  # hex64: interior nodes moved by up to 0.2 cell widths (seeded)


def workload(n, kind="cube64"):
    from emagddm_b200 import mesh
    if kind == "hex64":
        # On the unperturbed grid the ref tree takes every z-directed edge and
        # the z-directed coil current leaves F = 0; perturbed geometry keeps it.
        return mesh.perturbed(mesh.hex_scale(n), amplitude=HEX_AMPLITUDE, seed=n)
    return mesh.plain_scale(n)


def workload_config(n, n_dofs=None, nnz=None, kind="cube64"):
    if kind == "hex64":
        cfg = {"workload": f"hex{n}_iron_coil: {n}^3 HEX8_EDGE elements, interior nodes perturbed by up to "
                           f"{HEX_AMPLITUDE} cell (seed {n}), mu_r 1000 block, annulus coil J_z, ref tree gauge, "
                           f"FP64 GPU assembly (2x2x2 Gauss) + Jacobi-PCG to 1e-8",
               "n": n, "hexes": n ** 3, "gauge": "ref", "tol": TOL, "precond": "jacobi",
               "l2": "inputs larger than L2 (CSR values+indices > 126 MB), no flush"}
    else:
        cfg = {"workload": f"cube{n}_iron_coil: {n}^3 hex x 6 TET4_EDGE ({6 * n ** 3} tets), mu_r 1000 "
                           f"block, annulus coil J_z, ref tree gauge, FP64 GPU assembly + Jacobi-PCG "
                           f"to 1e-8",
               "n": n, "tets": 6 * n ** 3, "gauge": "ref", "tol": TOL, "precond": "jacobi",
               "l2": "inputs larger than L2 (CSR values+indices > 126 MB), no flush"}
    if n_dofs is not None:
        cfg["dofs"] = int(n_dofs)
    if nnz is not None:
        cfg["nnz"] = int(nnz)
        cfg["csr_bytes"] = int(12 * nnz + 4 * (n_dofs + 1))
    return cfg


class Clocks:
    """Samples SM clocks and throttle reasons through NVML while running."""

    def __init__(self, dev_index):
        self.samples, self.reasons, self.max_mhz = [], set(), None
        self._stop = threading.Event()
        self._t = None
        self.dev_index = dev_index

    def __enter__(self):
        try:
            import pynvml as N
            N.nvmlInit()
            h = N.nvmlDeviceGetHandleByIndex(self.dev_index)
            self.max_mhz = N.nvmlDeviceGetMaxClockInfo(h, N.NVML_CLOCK_SM)
            names = {getattr(N, k): k for k in dir(N) if k.startswith("nvmlClocksEventReason")
                     and isinstance(getattr(N, k), int)}

            def run():
                while not self._stop.is_set():
                    try:
                        self.samples.append(N.nvmlDeviceGetClockInfo(h, N.NVML_CLOCK_SM))
                        r = N.nvmlDeviceGetCurrentClocksEventReasons(h)
                        for bit, name in names.items():
                            if bit and (r & bit) == bit and name not in ("nvmlClocksEventReasonAll",):
                                self.reasons.add(name.replace("nvmlClocksEventReason", ""))
                    except Exception:
                        pass
                    self._stop.wait(0.1)
            self._t = threading.Thread(target=run, daemon=True)
            self._t.start()
        except Exception as e:  # NVML unavailable: report it
            self.reasons.add(f"nvml_unavailable:{type(e).__name__}")
        return self

    def __exit__(self, *a):
        self._stop.set()
        if self._t:
            self._t.join()

    def summary(self):
        return {"sm_mhz": statistics.median(self.samples) if self.samples else None,
                "sm_max_mhz": self.max_mhz, "samples": len(self.samples),
                "reasons": sorted(self.reasons)}


def measured_peak():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        return float(json.load(open(p))["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def ncu_traffic():
    """Per-launch DRAM bytes of the SpMV kernel from the committed ncu summary."""
    p = os.path.join(ROOT, "profiles", "cg_spmv_dot_cube64.md")
    try:
        for line in open(p):
            if line.startswith("traffic_bytes_per_launch_full:"):
                return float(line.split(":", 1)[1].split()[0])
    except OSError:
        pass
    return None


# --------------------------------------------------------------------------- ours
def bind_to_gpu_numa(local_rank):
    """Restrict this process to the host CPUs NVML reports as local to the
    GPU, so that the pinned host buffers of the end-to-end arm (allocated
    afterwards, first touch) sit on the GPU's NUMA node.  Returns a short
    description for the JSON line; leaves the affinity alone when NVML, the
    PCI lookup or the intersection with the allowed CPUs comes up empty."""
    import torch
    try:
        import pynvml as N
        p = torch.cuda.get_device_properties(local_rank)
        bus = "%08X:%02X:%02X.0" % (p.pci_domain_id, p.pci_bus_id, p.pci_device_id)
        N.nvmlInit()
        h = N.nvmlDeviceGetHandleByPciBusId(bus.encode())
        words = (os.cpu_count() + 63) // 64
        mask = N.nvmlDeviceGetCpuAffinity(h, words)
        local = {64 * w + b for w, m in enumerate(mask) for b in range(64) if (m >> b) & 1}
        cpus = local & os.sched_getaffinity(0)
        if not cpus:
            return "unbound (no GPU-local CPU allowed)"
        os.sched_setaffinity(0, cpus)
        return f"GPU-local NUMA CPUs ({len(cpus)})"
    except Exception as e:  # NVML missing or refused: measure unbound
        return f"unbound ({type(e).__name__})"


def run_ours(args, rank, world, local_rank):
    import torch

    from emagddm_b200 import _abi, api
    L = _abi.lib()
    dev = torch.device("cuda", local_rank)
    torch.cuda.set_device(dev)
    host_binding = bind_to_gpu_numa(local_rank)
    m = workload(args.n, args.workload)
    et = m.elem_type
    md = api.EMMeshData.from_cube(m)
    t0 = time.perf_counter()
    dm = api.EMDOFManager(md)
    dm.build()
    dm.applyTreeGauge(api.GaugeMode.REF)
    setup_dof_ms = (time.perf_counter() - t0) * 1e3
    l2g = np.ascontiguousarray(dm.getElemLocalToGlobal(), np.int32)
    n_dofs = int(l2g.max()) + 1
    xyz = np.ascontiguousarray(m.xyz, np.float64)
    tets = np.ascontiguousarray(m.tets, np.int32)
    mat = np.ascontiguousarray(m.material, np.int32)
    d_xyz, d_tets = torch.from_numpy(xyz).to(dev), torch.from_numpy(tets).to(dev)
    d_mat, d_l2g = torch.from_numpy(mat).to(dev), torch.from_numpy(l2g).to(dev)
    d_x = torch.empty(n_dofs, dtype=torch.float64, device=dev)
    # e2e inputs and result live in pinned host memory (page-locked copies)
    pinned = [torch.from_numpy(a).pin_memory() for a in (xyz, tets, mat, l2g)]
    p_xyz, p_tets, p_mat, p_l2g = (t.numpy() for t in pinned)
    h_x_t = torch.empty(n_dofs, dtype=torch.float64).pin_memory()
    h_x = h_x_t.numpy()
    stream = torch.cuda.current_stream(dev)
    sp = C.c_void_p(stream.cuda_stream)
    src, nsrc = _abi.sources_array(m.sources)
    srcp = C.cast(src, C.c_void_p)
    nu = np.ascontiguousarray(m.nu)
    sigma = np.ascontiguousarray(m.sigma)
    cfg = _abi.KrylovConfig(TOL, MAX_ITER, _abi.PRECOND_JACOBI)
    info = {}
    device_numbering = numbering_on_device(L, m, d_tets, l2g, stream, sp, dev)
    device_numbering["host_ms"] = setup_dof_ms

    if args.kernels_only:
        h = C.c_void_p()
        _abi.check(L.emg_system_create_typed(et, xyz.shape[0], C.c_void_p(d_xyz.data_ptr()), tets.shape[0],
                                             C.c_void_p(d_tets.data_ptr()), C.c_void_p(d_mat.data_ptr()),
                                             C.c_void_p(d_l2g.data_ptr()), n_dofs, 1, sp, C.byref(h)), "create")
        _abi.check(L.emg_system_assemble(h, _abi.ptr(nu), _abi.ptr(sigma), len(nu), srcp, nsrc, 0, sp),
                   "assemble")
        kt = (C.c_double * 3)()
        _abi.check(L.emg_cg_kernel_times(L.emg_system_matrix(h, 0), args.kernels_only, sp, kt), "times")
        L.emg_system_destroy(h)
        return {"mode": "kernels-only", "iterations": args.kernels_only,
                "cg_kernel_ms": {"spmv_dot": kt[0], "update": kt[1], "direction": kt[2]}}

    phase_log = []  # per step: host ms of create, assemble, solve, destroy; device ms of the solve

    ev_c = [torch.cuda.Event(enable_timing=True) for _ in range(4)]

    def step(resident: bool):
        t0 = time.perf_counter()
        ev_c[0].record(stream)
        h = C.c_void_p()
        if resident:
            rc = L.emg_system_create_typed(et, xyz.shape[0], C.c_void_p(d_xyz.data_ptr()), tets.shape[0],
                                           C.c_void_p(d_tets.data_ptr()), C.c_void_p(d_mat.data_ptr()),
                                           C.c_void_p(d_l2g.data_ptr()), n_dofs, 1, sp, C.byref(h))
        else:
            rc = L.emg_system_create_typed(et, p_xyz.shape[0], _abi.ptr(p_xyz), p_tets.shape[0], _abi.ptr(p_tets),
                                           _abi.ptr(p_mat), _abi.ptr(p_l2g), n_dofs, 0, sp, C.byref(h))
        _abi.check(rc, "emg_system_create")
        ev_c[1].record(stream)
        t1 = time.perf_counter()
        ev_c[2].record(stream)
        _abi.check(L.emg_system_assemble(h, _abi.ptr(nu), _abi.ptr(sigma), len(nu), srcp, nsrc, 0, sp),
                   "emg_system_assemble")
        ev_c[3].record(stream)
        t2 = time.perf_counter()
        out = _abi.Result()
        if resident:
            rc = L.emg_system_solve(h, 0, C.byref(cfg), C.c_void_p(d_x.data_ptr()), 1, sp, C.byref(out))
        else:
            rc = L.emg_system_solve(h, 0, C.byref(cfg), _abi.ptr(h_x), 0, sp, C.byref(out))
        if rc != 0:
            raise RuntimeError(f"solve status {rc}: {L.emg_last_error().decode()}")
        if "nnz" not in info:
            n_, nnz_ = C.c_int64(), C.c_int64()
            L.emg_system_info(h, C.byref(n_), C.byref(nnz_))
            info["nnz"] = nnz_.value
        info["iters"] = out.iterations
        info["res"] = out.residual_norm
        info["solve_ms"] = out.solve_time_ms
        t3 = time.perf_counter()
        L.emg_system_destroy(h)
        t4 = time.perf_counter()
        # host ms of create, assemble, solve, destroy; device ms of the solve, of
        # the create call (uploads + symbolic phase; host >> device places a
        # stall on the host side of the copies, device large on the DMA) and of
        # the numeric assembly
        phase_log.append([round((b - a) * 1e3, 2) for a, b in ((t0, t1), (t1, t2), (t2, t3), (t3, t4))]
                         + [round(out.solve_time_ms, 2), round(ev_c[0].elapsed_time(ev_c[1]), 2),
                            round(ev_c[2].elapsed_time(ev_c[3]), 3)])

    step_ms = {}

    def timed(resident, k, w):
        for _ in range(w):
            step(resident)
        barrier()
        torch.cuda.synchronize(dev)
        ev = [torch.cuda.Event(enable_timing=True) for _ in range(k + 1)]
        del phase_log[:]
        gc.collect()
        gc.disable()  # no collector pass inside the timed steps (they create no cycles)
        ev[0].record(stream)
        for i in range(k):
            step(resident)
            ev[i + 1].record(stream)
        torch.cuda.synchronize(dev)
        gc.enable()
        arm = "resident" if resident else "e2e"
        step_ms[arm] = [round(ev[i].elapsed_time(ev[i + 1]), 3) for i in range(k)]
        step_ms[arm + "_phases"] = list(phase_log)
        ms = ev[0].elapsed_time(ev[k])
        return max_over_ranks(ms)

    def barrier():
        if world > 1:
            import torch.distributed as dist
            dist.barrier()

    def max_over_ranks(v):
        if world == 1:
            return v
        import torch.distributed as dist
        t = torch.tensor([v], dtype=torch.float64, device=dev)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        return float(t.item())

    with Clocks(local_rank) as clk:
        total_ms = timed(True, args.steps, args.warmup)
    iters = info["iters"]
    total_e2e = timed(False, args.steps, args.warmup)
    e2e_iters = info["iters"]

    # roofline of the dominant kernel (SpMV + p.q of CG), live CUDA-event times
    h = C.c_void_p()
    _abi.check(L.emg_system_create_typed(et, xyz.shape[0], C.c_void_p(d_xyz.data_ptr()), tets.shape[0],
                                         C.c_void_p(d_tets.data_ptr()), C.c_void_p(d_mat.data_ptr()),
                                         C.c_void_p(d_l2g.data_ptr()), n_dofs, 1, sp, C.byref(h)), "create")
    _abi.check(L.emg_system_assemble(h, _abi.ptr(nu), _abi.ptr(sigma), len(nu), srcp, nsrc, 0, sp), "asm")
    kt = (C.c_double * 3)()
    Kh = L.emg_system_matrix(h, 0)
    _abi.check(L.emg_cg_kernel_times(Kh, 50, sp, kt), "kernel times")
    slots, slices = C.c_int64(), C.c_int64()
    L.emg_csr_solver_format(Kh, C.byref(slots), C.byref(slices))
    L.emg_system_destroy(h)
    # one instrumented step: host wall time of each phase (synchronized)
    phases = {}
    torch.cuda.synchronize(dev)
    t = time.perf_counter()
    h = C.c_void_p()
    L.emg_system_create_typed(et, xyz.shape[0], C.c_void_p(d_xyz.data_ptr()), tets.shape[0],
                              C.c_void_p(d_tets.data_ptr()), C.c_void_p(d_mat.data_ptr()),
                              C.c_void_p(d_l2g.data_ptr()), n_dofs, 1, sp, C.byref(h))
    torch.cuda.synchronize(dev)
    phases["create_symbolic"] = (time.perf_counter() - t) * 1e3
    t = time.perf_counter()
    L.emg_system_assemble(h, _abi.ptr(nu), _abi.ptr(sigma), len(nu), srcp, nsrc, 0, sp)
    torch.cuda.synchronize(dev)
    phases["assemble"] = (time.perf_counter() - t) * 1e3
    t = time.perf_counter()
    out = _abi.Result()
    L.emg_system_solve(h, 0, C.byref(cfg), C.c_void_p(d_x.data_ptr()), 1, sp, C.byref(out))
    torch.cuda.synchronize(dev)
    phases["solve"] = (time.perf_counter() - t) * 1e3
    phases["solve_device"] = out.solve_time_ms
    t = time.perf_counter()
    L.emg_system_destroy(h)
    phases["destroy"] = (time.perf_counter() - t) * 1e3
    nnz = info["nnz"]
    spmv_bytes = 12 * nnz + 4 * (n_dofs + 1) + 8 * n_dofs + 8 * n_dofs
    peak, peak_kind = measured_peak()
    achieved = spmv_bytes / (kt[0] * 1e-3) / 1e9
    # the committed capture covers the 64^3 TET4_EDGE matrix only
    traffic = ncu_traffic() if args.workload == "cube64" and args.n == 64 else None
    it_ms = sum(kt[:3])

    # numeric assembly: device time of the emg_system_assemble call in the
    # resident steps against its algorithmic bytes (elements, materials and
    # coordinates read once, K values and F written once)
    asm_ms = statistics.median(p[6] for p in step_ms["resident_phases"])
    asm_bytes = tets.nbytes + mat.nbytes + xyz.nbytes + 8 * nnz + 8 * n_dofs
    assembly = {"device_ms": asm_ms, "algorithmic_bytes": int(asm_bytes),
                "achieved_gbs": asm_bytes / (asm_ms * 1e-3) / 1e9,
                "frac_of_measured_hbm": asm_bytes / (asm_ms * 1e-3) / 1e9 / peak}

    ms_per_step = total_ms / args.steps
    value = world * args.steps / (total_ms * 1e-3)
    e2e_value = world * args.steps / (total_e2e * 1e-3)
    # per step: 23 launches of create + assemble + SELL build + Jacobi + CG
    # init (the committed launch list), the solution scatter, and the device
    # while-loop: bodies of 4 iterations x (SpMV, fused update) + 1 control
    bodies = -(-iters // 4)
    launches_per_step = 23 + 1 + bodies * (4 * 2 + 1)
    h2d = xyz.nbytes + tets.nbytes + mat.nbytes + l2g.nbytes
    line = {
        "metric": METRIC, "value": value, "unit": "solves/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_per_step,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": ("synthetic (structured hex grid, interior nodes perturbed, seed n; iron block + annulus coil)"
                 if args.workload == "hex64" else
                 "synthetic (seedless structured cube mesh; iron block + annulus coil)"),
        "config": {**workload_config(args.n, n_dofs, nnz, args.workload), "parallelism": f"replicas{world}",
                   "pcg_iterations": iters, "final_residual": info["res"],
                   "setup_dof_ms": setup_dof_ms, "device_numbering": device_numbering,
                   "cg_kernel_ms": {"spmv_dot": kt[0], "update": kt[1], "direction": kt[2]},
                   "cg_iteration_ms_kernels": it_ms,
                   "solve_ms": info["solve_ms"], "phase_ms": phases, "step_ms": step_ms, "assembly": assembly,
                   "median_step_ms": {a: statistics.median(step_ms[a]) for a in ("resident", "e2e")},
                   "solver_format": {"kind": "SELL-32-sigma4096", "slots": slots.value,
                                     "padding": slots.value / nnz - 1.0},
                   "host_cpus": host_binding,
                   "autotune": _abi.tune_report()},
        "clocks": clk.summary(),
        "e2e": {"value": e2e_value, "unit": "solves/s", "h2d_bytes_per_step": int(h2d),
                "d2h_bytes_per_step": int(h_x.nbytes), "ms_per_step": total_e2e / args.steps,
                "pcg_iterations": e2e_iters},
        "gpu_launches": int(launches_per_step * args.steps),
        "roofline": {"kernel": "k_cg_spmv_dot (CSR SpMV + p.q)", "bound": "hbm",
                     "achieved": achieved, "peak": peak, "peak_kind": peak_kind, "unit": "GB/s",
                     "frac": achieved / peak, "traffic": traffic,
                     "algorithmic_bytes_per_launch": spmv_bytes},
    }
    # the solution of the last timed (end-to-end) step, and the same system
    # solved again to 1e-12 for the tight comparison with the oracle
    x_tol = h_x.copy()
    h = C.c_void_p()
    _abi.check(L.emg_system_create_typed(et, xyz.shape[0], C.c_void_p(d_xyz.data_ptr()), tets.shape[0],
                                         C.c_void_p(d_tets.data_ptr()), C.c_void_p(d_mat.data_ptr()),
                                         C.c_void_p(d_l2g.data_ptr()), n_dofs, 1, sp, C.byref(h)), "create")
    _abi.check(L.emg_system_assemble(h, _abi.ptr(nu), _abi.ptr(sigma), len(nu), srcp, nsrc, 0, sp), "asm")
    out = _abi.Result()
    tight = _abi.KrylovConfig(1e-12, MAX_ITER, _abi.PRECOND_JACOBI)
    # the 1e-12 run may end on the reference's absolute breakdown test
    # (|p^T A p| < 1e-30, NUMERICAL_ERROR) or at MAX_ITER when the system's
    # rounding floor lies near 1e-12; its iterate is still the tight
    # comparison, reported with its status
    tight_rc = L.emg_system_solve(h, 0, C.byref(tight), _abi.ptr(h_x), 0, sp, C.byref(out))
    if tight_rc not in (_abi.EMG_SUCCESS, _abi.EMG_NUMERICAL_ERROR, _abi.EMG_MAX_ITER_REACHED):
        _abi.check(tight_rc, "tight solve")
    L.emg_system_destroy(h)
    x_tight, tight_iters = h_x.copy(), out.iterations
    line["config"]["tight_solve"] = {"status": int(tight_rc), "iterations": int(out.iterations),
                                     "residual": float(out.residual_norm)}
    csys = None
    if rank == 0 and not args.no_oracle:
        csys = cpu_system(m, l2g, n_dofs)
        line["config"]["oracle"] = oracle_check_plain(csys, x_tol, x_tight, tight_iters)
    if rank == 0 and not args.no_cpu_baseline:
        line["cpu_baseline"] = cpu_baseline(args, m, l2g, n_dofs, iters, csys)
    if rank == 0 and not args.no_comparison and args.workload == "cube64" and args.n == 64:
        line["config"]["comparison"] = metric_comparison(args, local_rank)
    return line


def rel_err(a, b):
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


def numbering_on_device(L, m, d_tets, l2g, stream, sp, dev):
    """The same DOF map computed by emg_dof_build_device from the device
    element array (edge IDs, free numbering, `ref` gauge): host wall time of
    the call (it synchronizes), median of 3 after one warm-up, and whether it
    equals the host numbering bit for bit."""
    import torch

    from emagddm_b200 import _abi
    d_dir = torch.from_numpy(np.ascontiguousarray(m.dirichlet, np.int32).reshape(-1)).to(dev)
    out = torch.empty(l2g.size, dtype=torch.int32, device=dev)
    ne, nf, nd = C.c_int64(), C.c_int64(), C.c_int64()
    ms = []
    for _ in range(4):
        torch.cuda.synchronize(dev)
        t0 = time.perf_counter()
        _abi.check(L.emg_dof_build_device(m.elem_type, m.n_nodes, m.n_tets, d_tets.data_ptr(), len(m.dirichlet),
                                          d_dir.data_ptr(), 0, _abi.GAUGE_REF, out.data_ptr(), C.byref(ne),
                                          C.byref(nf), C.byref(nd), sp), "emg_dof_build_device")
        ms.append((time.perf_counter() - t0) * 1e3)
    equal = bool(np.array_equal(out.cpu().numpy(), l2g.reshape(-1)))
    return {"ms": statistics.median(ms[1:]), "ms_runs": [round(x, 2) for x in ms], "equal_to_host": equal,
            "n_dofs": nd.value,
            "what": "emg_dof_build_device (GPU edge IDs, free numbering, ref tree-cotree gauge) from the device "
                    "element array; host_ms: the host numbering the timed steps use"}


def oracle_check_plain(csys, x_tol, x_tight, tight_iters):
    """The benchmarked system assembled and solved by the FP64 CPU oracle
    (restated reference assembly; the reference's CGSolver Jacobi iteration,
    iterative_solvers.cpp:424-503) on all host threads: one Jacobi-PCG run to
    1e-12 that also keeps the iterate at which a run to 1e-8 stops.  Reports
    the GPU's 1e-8 solution against the oracle's 1e-12 solution
    (oracle_rel_error, the solution bar) and against the oracle's own 1e-8
    iterate (same algorithm and stopping rule), the GPU's 1e-12 solution
    against the oracle's, and the true residual of the GPU solution on the
    oracle's matrix."""
    from oracle import oracle as O
    rp, col, kv, rhs, asm_ms = csys
    t0 = time.perf_counter()
    xo, st, it, res, xo_tol, it_tol = O.pcg_snap(rp, col, kv, rhs, tol=1e-12, snap_tol=TOL, max_iter=MAX_ITER,
                                                 precond=1)
    solve_ms = (time.perf_counter() - t0) * 1e3
    r = rhs - O.spmv(rp, col, kv, x_tol)
    return {"oracle_rel_error": rel_err(x_tol, xo),
            "oracle_rel_error_same_tolerance": rel_err(x_tol, xo_tol),
            "tight_rel_error": rel_err(x_tight, xo),
            "true_residual_on_oracle_matrix": float(np.linalg.norm(r) / np.linalg.norm(rhs)),
            "oracle_iterations": {"1e-8": it_tol, "1e-12": it}, "gpu_iterations_1e-12": tight_iters,
            "oracle_status": st, "oracle_residual": res, "threads": O.num_threads(),
            "assembly_ms": asm_ms, "solve_ms": solve_ms,
            "what": "GPU solution (Jacobi-PCG to 1e-8) vs the FP64 CPU oracle's Jacobi-PCG to 1e-12 on the "
                    "oracle's own assembly of the same mesh and DOF map"}


# ----------------------------------------------------------------- CPU side
def cpu_system(m, l2g, n_dofs):
    from oracle import oracle as O
    t0 = time.perf_counter()
    rp, col = O.pattern(l2g, n_dofs)
    rp, col, kv, _, rhs = O.assemble(m, l2g, n_dofs, rp=rp, col=col)
    return rp, col, kv, rhs, (time.perf_counter() - t0) * 1e3


def cpu_sample(m, l2g, n_dofs, iters_needed, sample_iters, csys=None):
    """Reference CGSolver (oracle/_ref) when built, else the oracle port:
    a bounded sample of iterations, projected to the full solve."""
    from oracle import oracle as O
    from oracle import refbridge as R
    rp, col, kv, rhs, asm_ms = csys if csys is not None else cpu_system(m, l2g, n_dofs)
    if R.available():
        _, st, it, res, setup_ms, solve_ms = R.krylov(0, rp, col, kv, rhs, tol=TOL,
                                                      max_iter=sample_iters, precond=1)
        kind, cores = "reference", 1
        what = (f"reference CGSolver+Jacobi (Eigen, 1 thread) set_matrix + {it} iterations on the same "
                f"system, projected to {iters_needed} iterations; assembly by the restated oracle "
                f"(1 thread; the reference's TET4_EDGE integrator returns zeros)")
    else:
        t0 = time.perf_counter()
        _, st, it, res = O.pcg(rp, col, kv, rhs, tol=TOL, max_iter=sample_iters, precond=1)
        solve_ms, setup_ms = (time.perf_counter() - t0) * 1e3, 0.0
        kind, cores = "port", O.num_threads()
        what = f"oracle port Jacobi-PCG, {it} iterations, projected to {iters_needed}"
    per_iter = solve_ms / max(it, 1)
    total_ms = asm_ms + setup_ms + per_iter * iters_needed
    return total_ms, {"kind": kind, "cores": cores, "sample": what,
                      "assembly_ms": asm_ms, "set_matrix_ms": setup_ms, "ms_per_iteration": per_iter,
                      "projected_ms_per_solve": total_ms}


def cpu_baseline(args, m, l2g, n_dofs, iters, csys=None):
    total_ms, d = cpu_sample(m, l2g, n_dofs, iters, args.cpu_iters, csys)
    return {"value": 1e3 / total_ms, "unit": "solves/s", **d}


def batch_measure(n_inst, steps, warmup, local_rank, plain_stride, oracle_stride, clocks=None):
    """512 independent instances (n ~ U{8..32}, seed 7+i): one block-diagonal
    system, lockstep Jacobi-PCG to 1e-8 in one device loop, `steps` timed
    steps after `warmup` (assembly + solve per step, inputs resident), first
    with the built-in launch configuration, then the autotuned one; the same
    instances solved one at a time through emg_system_solve (every
    `plain_stride`-th, projected) and the per-instance error of every
    `oracle_stride`-th against the FP64 CPU oracle.  Returns (tuned ms per
    step, config dict)."""
    import torch

    from emagddm_b200 import _abi, batch
    from oracle import oracle as O
    L = _abi.lib()
    dev = torch.device("cuda", local_rank)
    torch.cuda.set_device(dev)
    t0 = time.perf_counter()
    inst = batch.make_instances(n_inst)
    b = batch.build_batch(inst)
    setup_ms = (time.perf_counter() - t0) * 1e3
    res_d = {k: torch.from_numpy(getattr(b, k)).to(dev) for k in ("xyz", "tets", "material", "l2g")}
    ptrs = {k: C.c_void_p(v.data_ptr()) for k, v in res_d.items()}
    x = torch.zeros(b.n_rows, dtype=torch.float64, device=dev)
    stream = torch.cuda.current_stream(dev)
    info = {}

    def step():
        S = batch.BatchSystem(b, resident=ptrs)
        rc, res = S.solve(x.data_ptr(), tol=TOL, max_iter=MAX_ITER)
        if rc != 0:
            raise RuntimeError(f"batch status {rc}: {L.emg_last_error().decode()}")
        info["res"] = res
        del S

    def timed_steps():
        for _ in range(warmup):
            step()
        torch.cuda.synchronize(dev)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(steps):
            step()
        e1.record(stream)
        torch.cuda.synchronize(dev)
        return e0.elapsed_time(e1) / steps

    # the built-in launch configuration first (autotuner off), then the tuned one
    L.emg_tune_enable(0)
    ms_default = timed_steps()
    L.emg_tune_enable(1)
    if clocks is not None:
        with clocks:
            ms = timed_steps()
    else:
        ms = timed_steps()
    iters = [r["iterations"] for r in info["res"]]
    # plain path: the same instances one at a time (a sample, projected)
    sample = list(range(0, len(inst), plain_stride))
    t_plain = 0.0
    for k in sample:
        m = inst[k]
        xs, ts, ms_, ls = (np.ascontiguousarray(m.xyz), np.ascontiguousarray(m.tets, np.int32),
                           np.ascontiguousarray(m.material, np.int32), b.l2g_each[k])
        torch.cuda.synchronize(dev)
        ta = time.perf_counter()
        h = C.c_void_p()
        _abi.check(L.emg_system_create(xs.shape[0], _abi.ptr(xs), ts.shape[0], _abi.ptr(ts), _abi.ptr(ms_),
                                       _abi.ptr(ls), 0, None, C.byref(h)), "create")
        arr, ns = _abi.sources_array(m.sources)
        L.emg_system_assemble(h, _abi.ptr(m.nu), _abi.ptr(m.sigma), len(m.nu), C.cast(arr, C.c_void_p), ns, 0,
                              None)
        out = _abi.Result()
        cfg = _abi.KrylovConfig(TOL, MAX_ITER, _abi.PRECOND_JACOBI)
        xh = np.empty(int(b.block_row_ptr[k + 1] - b.block_row_ptr[k]))
        L.emg_system_solve(h, 0, C.byref(cfg), _abi.ptr(xh), 0, None, C.byref(out))
        L.emg_system_destroy(h)
        t_plain += time.perf_counter() - ta
    plain_per_inst_ms = t_plain / len(sample) * 1e3
    # per-instance error against the FP64 CPU oracle (its own assembly and a
    # Jacobi-PCG solve to 1e-12)
    xs_all = x.cpu().numpy()
    errs, t0 = [], time.perf_counter()
    oracle_sample = list(range(0, len(inst), oracle_stride))
    for k in oracle_sample:
        m = inst[k]
        r0, r1 = int(b.block_row_ptr[k]), int(b.block_row_ptr[k + 1])
        orp, ocol, okv, _, orhs = O.assemble(m, b.l2g_each[k], r1 - r0)
        xo, st, it, _ = O.pcg(orp, ocol, okv, orhs, tol=1e-12, max_iter=MAX_ITER, precond=1)
        errs.append(float(np.linalg.norm(xs_all[r0:r1] - xo) / max(np.linalg.norm(xo), 1e-300)))
    oracle_ms = (time.perf_counter() - t0) * 1e3
    value = len(inst) / (ms * 1e-3)
    cfg = {"workload": f"batch{len(inst)}: n~U{{8..32}} cubes x 6 tets, random mu_r box, "
                       f"J_z sub-box, ref tree gauge, Jacobi-PCG to 1e-8, one lockstep device loop",
           "instances": len(inst), "rows": b.n_rows, "tets": int(b.tets.shape[0]),
           "steps": steps, "warmup": warmup, "ms_per_step": ms, "solves_per_s": value,
           "iterations_min_median_max": [min(iters), int(np.median(iters)), max(iters)],
           "setup_ms": setup_ms,
           "plain_one_at_a_time": {"ms_per_instance": plain_per_inst_ms,
                                   "solves_per_s": 1e3 / plain_per_inst_ms,
                                   "sample": len(sample)},
           "batched_vs_plain": value / (1e3 / plain_per_inst_ms),
           "oracle_rel_error_sample_max": max(errs), "oracle_rel_error_sample_median": float(np.median(errs)),
           "oracle_sample": len(errs), "oracle_sample_instances": f"every {oracle_stride}th",
           "oracle_ms": oracle_ms, "oracle_threads": O.num_threads(),
           "autotune": {"ms_per_step_default": ms_default, "ms_per_step_tuned": ms,
                        "tuned_vs_default": ms_default / ms}}
    return ms, cfg


def run_batch(args, rank, world, local_rank):
    """The batched many-instance workload as its own line (batch_measure);
    value = instance solves per second over all ranks."""
    from emagddm_b200 import _abi
    clk = Clocks(local_rank)
    ms, cfg = batch_measure(args.instances, args.steps, args.warmup, local_rank,
                            plain_stride=max(1, args.instances // 16), oracle_stride=max(1, args.instances // 32),
                            clocks=clk)
    cfg["autotune"]["decisions"] = _abi.tune_report()
    value = world * cfg["instances"] / (ms * 1e-3)
    return {
        "metric": METRIC + " [batched many-instance]", "value": value, "unit": "solves/s",
        "n_gpus": world, "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic (seeded random instances, seed 7+i)",
        "config": cfg,
        "clocks": clk.summary(),
    }


FLAG_FACTOR_TF32 = 16
FETI_VARIANTS = {
    "fp64": ("FP64 factor, deluxe-scaled Dirichlet preconditioner with FP64 blocks", 2, 0),
    "fp32_precond": ("FP64 factor, deluxe preconditioner blocks read in FP32", 3, 0),
    "tf32_factor": ("mixed-precision factor: update-block and pivot-column contractions on the tcgen05 tensor "
                    "cores (two-term TF32, FP32 accumulation), FP64 refinement on the true residual",
                    2, FLAG_FACTOR_TF32),
    "tf32_factor_fp32_precond": ("mixed-precision factor and FP32 preconditioner blocks", 3, FLAG_FACTOR_TF32),
}


def fetidp_variants(fd, names, steps, warmup, stream, dev):
    """factor + solve to a true residual of 1e-8 for each variant (CUDA
    events around the pair, mean over `steps` after `warmup` untimed pairs)."""
    import torch
    from emagddm_b200 import _abi
    L = _abi.lib()
    res = {}
    x = None
    for name in names:
        what, precond, flags = FETI_VARIANTS[name]
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        per, st, failed = [], None, None
        for k in range(warmup + steps):
            e0.record(stream)
            rc = fd.factor(flags=flags)
            if rc:
                raise RuntimeError(f"factor {rc}: {L.emg_last_error().decode()}")
            x, rc, r = fd.solve(tol=TOL, max_iter=2000, precond=precond)
            e1.record(stream)
            torch.cuda.synchronize(dev)
            if rc:  # a variant that does not reach the tolerance is reported, not timed
                failed = {"status": rc, "error": L.emg_last_error().decode(), **fd.stats()}
                break
            if k >= warmup:
                per.append(e0.elapsed_time(e1))
                st = fd.stats()
        if failed:
            res[name] = {"what": what, "failed": failed}
            continue
        its = max(int(st["iterations"]), 1)
        # dense blocks read per multiplier iteration: L^-1 (lower part, then
        # the stored transpose: the whole n_D^2 block once), the S_DD tiles on
        # and below the diagonal and the four deluxe blocks of every face
        # (FP32 copies of both with the FP32 preconditioner)
        fi = fd.info()
        pw = 4 if precond == 3 else 8
        nb = fi["dual_block_doubles"] * 8 + fi["sym_tile_doubles"] * pw + 4 * fi["face_block_doubles"] * pw
        peak, _ = measured_peak()
        per_it = st["lambda_ms"] / its
        res[name] = {"what": what, "ms": statistics.mean(per), "ms_steps": [round(v, 3) for v in per],
                     "factor_ms": st["factor_ms"], "solve_ms": st["solve_ms"],
                     "lambda_iterations": int(st["iterations"]), "passes": int(st["passes"]),
                     "true_residual": st["residual"],
                     "solve_phases_ms": {"lambda_iterations": st["lambda_ms"], "front_solves": st["fronts_ms"]},
                     "lambda_iteration": {"ms": per_it, "dense_block_bytes": nb,
                                          "achieved_gbs": nb / (per_it * 1e-3) / 1e9,
                                          "frac_of_measured_hbm": nb / (per_it * 1e-3) / 1e9 / peak},
                     "_x": x}
    return res


def pcg_same_gauge(m, l2g, n_dofs, tols, dev):
    """Jacobi-PCG (the plain GPU path) on the partition-gauged system, through
    the host-buffer C ABI: assembly + solve per tolerance."""
    import torch
    from emagddm_b200 import _abi
    L = _abi.lib()
    xs, ts, mt = (np.ascontiguousarray(m.xyz), np.ascontiguousarray(m.tets, np.int32),
                  np.ascontiguousarray(m.material, np.int32))
    l2g = np.ascontiguousarray(l2g, np.int32)
    h = C.c_void_p()
    _abi.check(L.emg_system_create(xs.shape[0], _abi.ptr(xs), ts.shape[0], _abi.ptr(ts), _abi.ptr(mt),
                                   _abi.ptr(l2g), 0, None, C.byref(h)), "create")
    arr, ns = _abi.sources_array(m.sources)
    out, sols = {}, {}
    try:
        for tol in tols:
            xp = np.empty(n_dofs)
            cfg = _abi.KrylovConfig(tol, 400000, _abi.PRECOND_JACOBI)
            r = _abi.Result()
            torch.cuda.synchronize(dev)
            ta = time.perf_counter()
            L.emg_system_assemble(h, _abi.ptr(m.nu), _abi.ptr(m.sigma), len(m.nu), C.cast(arr, C.c_void_p), ns, 0,
                                  None)
            L.emg_system_solve(h, 0, C.byref(cfg), _abi.ptr(xp), 0, None, C.byref(r))
            out[f"{tol:g}"] = {"ms": (time.perf_counter() - ta) * 1e3, "iterations": r.iterations,
                               "status": r.status, "residual": r.residual_norm}
            sols[tol] = xp
    finally:
        L.emg_system_destroy(h)
    return out, sols


def metric_comparison(args, local_rank):
    """The metric's own comparison on the 64-subdomain configuration: the
    64^3 plain-at-scale problem split into 4^3 jittered boxes (seed
    20261203), partition tree gauge, time to a true FP64 relative residual of
    1e-8 for plain FETI-DP and each built addition, next to the plain GPU
    Jacobi-PCG on the same gauged system; the FETI-DP solution is checked on
    the oracle's own FP64 assembly (true residual) and against a GPU
    Jacobi-PCG solve to 1e-12."""
    import torch

    from emagddm_b200 import _abi, fetidp, mesh
    from oracle import oracle as O
    dev = torch.device("cuda", local_rank)
    stream = torch.cuda.current_stream(dev)
    m = workload(64)
    t0 = time.perf_counter()
    part = mesh.jittered_partition(m, 4)
    fd = fetidp.FetiDP(m, part, 64)
    setup_ms = (time.perf_counter() - t0) * 1e3
    info = fd.info()
    names = [v for v in args.feti_variants.split(",") if v in FETI_VARIANTS]
    if "fp64" not in names:
        names.insert(0, "fp64")
    var = fetidp_variants(fd, names, steps=3, warmup=2, stream=stream, dev=dev)
    x_feti = var["fp64"].pop("_x")
    for v in var.values():
        v.pop("_x", None)
    timed = {k: v for k, v in var.items() if "ms" in v}
    n_dofs = fd.map.n_dofs
    pcg, sols = pcg_same_gauge(m, fd.map.l2g, n_dofs, (TOL, 1e-12), dev)
    orp, ocol, okv, _, orhs = O.assemble(m, fd.map.l2g, n_dofs)
    r = orhs - O.spmv(orp, ocol, okv, x_feti)
    del fd
    learned = comparison_learned(args, local_rank) if args.cmp_train_fields > 0 else None
    batched = None
    if args.cmp_batch_instances > 0:  # the batched many-instance addition, reduced to 2 timed steps
        n_b = args.cmp_batch_instances
        _, batched = batch_measure(n_b, steps=2, warmup=1, local_rank=local_rank, plain_stride=max(1, n_b // 16),
                                   oracle_stride=max(1, n_b // 16))
    plain_fetidp = var["fp64"]["ms"]
    plain_pcg = pcg[f"{TOL:g}"]["ms"]
    best = min(timed, key=lambda k: timed[k]["ms"])
    return {
        "workload": "fetidp64: cube64_iron_coil split into 64 jittered box subdomains (seed 20261203), partition "
                    "tree gauge, time to a true FP64 relative residual of 1e-8",
        "dofs": n_dofs, "n_lambda": info["n_lambda"], "n_coarse": info["n_coarse"],
        "setup_host_ms": setup_ms, "fetidp": var, "plain_pcg_same_gauge": pcg,
        "learned": learned,
        "batched": batched,
        "combination": "mixed factor + learned + graph loop: not run, the mixed-precision factor does not converge "
                       "at 64^3 (fetidp.tf32_factor above)",
        "best": best, "best_ms": var[best]["ms"],
        "speedup_vs_plain_fetidp": plain_fetidp / var[best]["ms"],
        "speedup_vs_plain_pcg": plain_pcg / var[best]["ms"],
        "plain_fetidp_vs_plain_pcg": plain_pcg / plain_fetidp,
        "target": "additions >= 5x faster than the plain GPU FETI-DP/PCG path",
        "autotune": _abi.tune_report(),
        "oracle": {"true_residual_on_oracle_matrix": float(np.linalg.norm(r) / np.linalg.norm(orhs)),
                   "rel_diff_vs_gpu_pcg_1e-12": rel_err(x_feti, sols[1e-12]),
                   "what": "FP64 FETI-DP solution: residual on the CPU oracle's own assembly of the partition-"
                           "gauged system, and difference from the GPU Jacobi-PCG solution to 1e-12"},
    }


def comparison_learned(args, local_rank):
    """The learned interface preconditioner on its own configuration (64^3,
    64 jittered boxes, random log-normal mu_r fields, curl-T sources), with a
    reduced training set so that it fits the default run: training pairs from
    `cmp_train_fields` fields (seeds 1000+), 20 epochs, then `cmp_eval_fields`
    held-out fields (seeds 2000+) solved with deluxe alone and deluxe +
    learned (flexible CG) to a true residual of 1e-8."""
    import torch

    from emagddm_b200 import learned
    t0 = time.perf_counter()
    tr = learned.Trainer(n=64, parts=4, seed=1)
    R, T = [], []
    for k in range(args.cmp_train_fields):
        r, t = tr.pairs(np.random.default_rng(1000 + k), per_solve=8, stride=3)
        R += r
        T += t
    losses = tr.train(R, T, epochs=20, batch=32, lr=1e-3)
    torch.cuda.synchronize()
    prep_ms = (time.perf_counter() - t0) * 1e3
    rows = []
    for k in range(args.cmp_eval_fields):
        o = tr.evaluate(np.random.default_rng(2000 + k), tol=TOL)
        rows.append((o[2]["iterations"], o[4]["iterations"], o[2]["ms"], o[4]["ms"], o[2]["residual"],
                     o[4]["residual"], o[2]["status"], o[4]["status"]))
    a = np.array(rows, dtype=float)
    return {"what": "deluxe vs deluxe + learned MLP correction (flexible CG), random mu_r fields; reduced training "
                    "set (the learned64 workload trains on 200 fields)",
            "train_fields": args.cmp_train_fields, "pairs": len(R), "eval_fields": args.cmp_eval_fields,
            "prep_ms": prep_ms, "loss_first_last": [losses[0], losses[-1]],
            "iterations_mean": {"deluxe": a[:, 0].mean(), "deluxe_plus_learned": a[:, 1].mean()},
            "solve_ms_mean": {"deluxe": a[:, 2].mean(), "deluxe_plus_learned": a[:, 3].mean()},
            "true_residual_max": {"deluxe": a[:, 4].max(), "deluxe_plus_learned": a[:, 5].max()},
            "all_converged": bool((a[:, 6] == 0).all() and (a[:, 7] == 0).all()),
            "learned_vs_deluxe_time": a[:, 2].mean() / a[:, 3].mean()}


def run_fetidp(args, rank, world, local_rank):
    """FETI-DP on the 64^3 plain-at-scale problem split into parts^3 box
    subdomains by jittered cut planes (seed 20261203), partition tree gauge.
    One step = numeric factorization (union assembly, multifrontal K_rr,
    S_DD and its inverse factor, coarse matrix, deluxe weights) + solve to a
    true relative residual of 1e-8.  Beside it: Jacobi-PCG on the same gauged
    system (assembly + solve), and the difference of the two solutions."""
    import torch

    from emagddm_b200 import fetidp, mesh
    dev = torch.device("cuda", local_rank)
    torch.cuda.set_device(dev)
    from emagddm_b200 import _abi
    m = workload(args.n)
    part = mesh.jittered_partition(m, args.parts)
    stream = torch.cuda.current_stream(dev)
    default = None
    if not args.mixed:  # the built-in solve-kernel widths (autotuner off) on a solver of their own
        _abi.lib().emg_tune_enable(0)
        fd0 = fetidp.FetiDP(m, part, args.parts ** 3)
        default = fetidp_variants(fd0, ["fp64"], steps=args.steps, warmup=args.warmup, stream=stream, dev=dev)["fp64"]
        default.pop("_x", None)
        del fd0
        _abi.lib().emg_tune_enable(1)
    t0 = time.perf_counter()
    fd = fetidp.FetiDP(m, part, args.parts ** 3)
    setup_ms = (time.perf_counter() - t0) * 1e3
    info = fd.info()
    name = {(2, 0): "fp64", (3, 0): "fp32_precond", (2, 1): "tf32_factor",
            (3, 1): "tf32_factor_fp32_precond"}.get((args.feti_precond, int(args.mixed)))
    if name is None:
        raise SystemExit(f"--feti-precond {args.feti_precond}: use 2 or 3")
    with Clocks(local_rank) as clk:
        v = fetidp_variants(fd, [name], steps=args.steps, warmup=args.warmup, stream=stream, dev=dev)[name]
    if "failed" in v:  # reported in the line (value null), not an abort
        return {"metric": METRIC + " [FETI-DP]", "value": None, "unit": "solves/s", "n_gpus": world,
                "steps": args.steps, "warmup": args.warmup, "ms_per_step": None, "higher_is_better": True,
                "scaling": "weak", "vs_baseline": None, "dtype": "f64",
                "config": {"workload": f"fetidp{args.n}", "n": args.n, "subdomains": args.parts ** 3,
                           "variant": v, "plan": info}, "clocks": clk.summary()}
    x = v.pop("_x")
    ms = v["ms"]
    pcg, sols = pcg_same_gauge(m, fd.map.l2g, fd.map.n_dofs, (TOL, 1e-12), dev)
    value = world * 1e3 / ms
    return {
        "metric": METRIC + " [FETI-DP]", "value": value, "unit": "solves/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic (structured cube, jittered box partition seed 20261203)",
        "config": {"workload": f"fetidp{args.n}: cube{args.n}_iron_coil split into {args.parts ** 3} jittered box "
                               f"subdomains, partition tree gauge, FETI-DP (multifrontal K_rr, deluxe-scaled "
                               f"Dirichlet preconditioner, defect correction) to a true residual of 1e-8",
                   "n": args.n, "subdomains": args.parts ** 3, "setup_host_ms": setup_ms,
                   "variant": v, "plan": info,
                   "device_gb": 8e-9 * (info["factor_doubles"] + info["update_pool_doubles"]
                                        + 2 * info["dual_block_doubles"]),
                   "plain_pcg_same_gauge": pcg, "rel_diff_vs_pcg_1e-12": rel_err(x, sols[1e-12]),
                   "fetidp_vs_plain_pcg": pcg[f"{TOL:g}"]["ms"] / ms,
                   "autotune": {"decisions": _abi.tune_report(),
                                "default_widths": {k: default[k] for k in ("ms", "factor_ms", "solve_ms",
                                                                           "solve_phases_ms")} if default else None,
                                "tuned_vs_default": default["ms"] / ms if default else None}},
        "clocks": clk.summary(),
    }


def run_learned(args, rank, world, local_rank):
    """Learned interface preconditioner on the 64-subdomain FETI-DP setup:
    random log-normal mu_r fields (GRF, corr 0.1, sigma 1.5, mu_r in
    [1, 2000]) and divergence-free J = curl T (corr 0.15).  Training pairs
    from `train_fields` fields (seeds 1000+), evaluation on `eval_fields`
    held-out fields (seeds 2000+): iterations and solve time to a true
    residual of 1e-8, deluxe Dirichlet vs deluxe + learned (flexible CG)."""
    import torch

    from emagddm_b200 import learned
    torch.cuda.set_device(local_rank)
    t0 = time.perf_counter()
    tr = learned.Trainer(n=args.n, parts=args.parts, seed=1)
    setup_ms = (time.perf_counter() - t0) * 1e3
    R, T = [], []
    t0 = time.perf_counter()
    for k in range(args.train_fields):
        r, t = tr.pairs(np.random.default_rng(1000 + k), per_solve=8, stride=3)
        R += r
        T += t
    pairs_ms = (time.perf_counter() - t0) * 1e3
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    losses = tr.train(R, T, epochs=20, batch=32, lr=1e-3)
    torch.cuda.synchronize()
    train_ms = (time.perf_counter() - t0) * 1e3
    rows = []
    with Clocks(local_rank) as clk:
        for k in range(args.eval_fields):
            o = tr.evaluate(np.random.default_rng(2000 + k), tol=TOL)
            rows.append((o[2]["iterations"], o[4]["iterations"], o[2]["ms"], o[4]["ms"], o[2]["residual"],
                         o[4]["residual"], o[2]["status"], o[4]["status"]))
    a = np.array(rows, dtype=float)
    plain_ms, learn_ms = a[:, 2].mean(), a[:, 3].mean()
    return {
        "metric": METRIC + " [learned interface preconditioner]", "value": 1e3 / learn_ms, "unit": "solves/s",
        "n_gpus": world, "steps": args.eval_fields, "warmup": 0, "ms_per_step": learn_ms, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64 (MLP bf16 weights, fp32 accumulate)",
        "data": "synthetic (GRF mu_r fields, curl-T sources; seeds 1000+ / 2000+)",
        "config": {"workload": f"learned{args.n}: cube{args.n} split into {args.parts ** 3} jittered boxes, per-subdomain "
                               f"3-layer MLP (width 256) correcting the deluxe Dirichlet preconditioner in flexible "
                               f"CG, solves to a true residual of 1e-8",
                   "train_fields": args.train_fields, "pairs": len(R), "eval_fields": args.eval_fields,
                   "setup_host_ms": setup_ms, "pair_generation_ms": pairs_ms, "train_ms": train_ms,
                   "loss_first_last": [losses[0], losses[-1]],
                   "iterations_mean": {"deluxe": a[:, 0].mean(), "deluxe_plus_learned": a[:, 1].mean()},
                   "solve_ms_mean": {"deluxe": plain_ms, "deluxe_plus_learned": learn_ms},
                   "true_residual_max": {"deluxe": a[:, 4].max(), "deluxe_plus_learned": a[:, 5].max()},
                   "all_converged": bool((a[:, 6] == 0).all() and (a[:, 7] == 0).all()),
                   "learned_vs_deluxe_time": plain_ms / learn_ms},
        "clocks": clk.summary(),
    }


def run_reference(args):
    from oracle import oracle as O
    m = workload(args.n)
    dof = O.dof_build(m.tets, m.dirichlet, gauge=O.GAUGE_REF)
    l2g = dof["l2g"]
    n_dofs = int(l2g.max()) + 1
    rp, col, kv, rhs, _ = cpu_system(m, l2g, n_dofs)
    # iterations to 1e-8 of this system, from the oracle port on all host threads
    _, st, iters_needed, _ = O.pcg(rp, col, kv, rhs, tol=TOL, max_iter=MAX_ITER, precond=1)
    vals = []
    d = None
    for k in range(args.warmup + args.steps):
        total_ms, d = cpu_sample(m, l2g, n_dofs, iters_needed, args.cpu_iters)
        if k >= args.warmup:
            vals.append(total_ms)
    ms = statistics.mean(vals)
    v = 1e3 / ms
    return {"impl": "reference", "metric": METRIC, "value": v, "unit": "solves/s", "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {**workload_config(args.n, n_dofs, int(rp[-1])), "pcg_iterations": iters_needed},
            "cpu_baseline": {"value": v, **d},
            "e2e": {"value": v, "unit": "solves/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}


def main():
    args = parse()
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        if rank == 0:
            print(json.dumps(run_reference(args)), flush=True)
        return
    if world > 1:
        import datetime

        import torch
        import torch.distributed as dist
        torch.cuda.set_device(local_rank)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300),
                                device_id=torch.device("cuda", local_rank))
    try:
        if args.workload == "batch512":
            line = run_batch(args, rank, world, local_rank)
        elif args.workload == "fetidp64":
            line = run_fetidp(args, rank, world, local_rank)
        elif args.workload == "learned64":
            line = run_learned(args, rank, world, local_rank)
        else:
            line = run_ours(args, rank, world, local_rank)
        if rank == 0:
            print(json.dumps(line), flush=True)
    finally:
        if world > 1:
            import torch.distributed as dist
            dist.destroy_process_group()


if __name__ == "__main__":
    main()
