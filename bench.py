#!/usr/bin/env python
"""Benchmark of the solid-mechanics Newton step on the 100^3 hex8 J2 mesh (3,090,903 DOFs).

Metric (one JSON line on rank 0): hex8 elements assembled per second, where one assembly is the
full fused pass that neon splits over update_internal_variables + assemble_stiffness +
compute_internal_force: deformation measures, the J2 return mapping at all 8,000,000 quadrature
points (plastic state), the tangent stiffness scattered into the 245,438,109-entry CSR pattern and
the internal force.  A step = one assembly with inputs resident in HBM (K, state and pattern are
far larger than L2, so no flush is needed).  Reported beside it: the Newton-step time of the
FP64 and mixed-precision device paths over the first load increments of the cyclic history and
the relative displacement error of the mixed path against the FP64 path, and the batched
workload (256 tet4 neo-Hooke boxes of uneven size in one context).

    python bench.py [--gpus N --steps K --warmup W] [--impl reference]

Under torchrun each rank runs an independent replica (the problem does not shard across GPUs);
``value`` sums the ranks' elements over the slowest rank's time.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

# reliable-update interval of the mixed Newton path: the FP32 residual is replaced by the FP64
# one after each 1/100 reduction (C3 first two increments: 12,557 CG iterations against 14,418
# at 1e-3 and 12,608 for FP64; C2 first increment: 6,174 against 6,325 and 6,115)
MIXED_DELTA = 1e-2
METRIC = "hex8 elements assembled/s + Newton-step s @3M DOF: mixed vs FP64 GPU, err<=1e-8"
UNIT = "elements/s"


_T0 = time.perf_counter()


def log(msg):
    """Progress on stderr (the JSON line alone goes to stdout)."""
    print(f"[bench {time.perf_counter() - _T0:8.1f}s] {msg}", file=sys.stderr, flush=True)


def max_over_ranks(t, dist, device="cuda"):
    """The slowest rank's time (every rank gets it); t itself when not distributed."""
    if dist is None:
        return t
    import torch
    tt = torch.tensor([float(t)], dtype=torch.float64, device=device)
    dist.all_reduce(tt, op=dist.ReduceOp.MAX)
    return float(tt.item())


def _env_int(k, d):
    try:
        return int(os.environ.get(k, d))
    except ValueError:
        return d


def plastic_displacement(mesh, level=2.5e-3):
    """A displacement field well past first yield: uniaxial z stretch with a shear twist."""
    X = mesh.X
    u = np.zeros(3 * mesh.num_nodes)
    u[2::3] = level * X[:, 2]
    u[0::3] = 0.3 * level * X[:, 2] * (X[:, 1] - 0.5)
    u[1::3] = -0.3 * level * X[:, 2] * (X[:, 0] - 0.5)
    return u


class ClockSampler:
    """SM clocks and clock-event reasons during the timed region, read (never set) through NVML
    from a thread polling every 5 ms, with one sample at start and one at stop, so that even a
    timed region of a few tens of milliseconds has samples; `nvidia-smi -lms 200` as the
    fallback when NVML is not importable."""
    QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
    REASONS = (("sw_power_cap", 0x4), ("hw_slowdown", 0x8), ("sw_thermal_slowdown", 0x20),
               ("hw_thermal_slowdown", 0x40))

    def __init__(self, index=0):
        self.index = index
        self.proc = None
        self.nvml = None
        self.lines = []
        self.samples = []  # (sm MHz, max sm MHz, reasons bitmask)
        self.stop_event = threading.Event()

    def _nvml_sample(self):
        nv, h = self.nvml
        try:
            sm = nv.nvmlDeviceGetClockInfo(h, nv.NVML_CLOCK_SM)
            smax = nv.nvmlDeviceGetMaxClockInfo(h, nv.NVML_CLOCK_SM)
            reasons = nv.nvmlDeviceGetCurrentClocksEventReasons(h) \
                if hasattr(nv, "nvmlDeviceGetCurrentClocksEventReasons") \
                else nv.nvmlDeviceGetCurrentClocksThrottleReasons(h)
            self.samples.append((float(sm), float(smax), int(reasons)))
        except Exception:  # a failed read leaves a gap, not an error
            pass

    def _poll(self):
        while not self.stop_event.wait(0.005):
            self._nvml_sample()

    def start(self):
        try:
            import pynvml as nv
            nv.nvmlInit()
            bus = None
            try:
                import torch
                pr = torch.cuda.get_device_properties(torch.cuda.current_device())
                bus = f"{pr.pci_domain_id:08X}:{pr.pci_bus_id:02X}:{pr.pci_device_id:02X}.0"
            except Exception:
                bus = None
            h = nv.nvmlDeviceGetHandleByPciBusId(bus) if bus else \
                nv.nvmlDeviceGetHandleByIndex(self.index)
            self.nvml = (nv, h)
            self._nvml_sample()
            self.thread = threading.Thread(target=self._poll, daemon=True)
            self.thread.start()
            return
        except Exception:
            self.nvml = None
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.index), f"--query-gpu={self.QUERY}",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except (OSError, FileNotFoundError):
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if self.nvml is not None:
            self.stop_event.set()
            self.thread.join(timeout=5)
            self._nvml_sample()
            sm = [x[0] for x in self.samples]
            smax = max((x[1] for x in self.samples), default=None)
            reasons = sorted({name for _, _, m in self.samples for name, bit in self.REASONS
                              if m & bit})
            try:
                self.nvml[0].nvmlShutdown()
            except Exception:
                pass
            return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": smax,
                    "reasons": reasons, "samples": len(sm), "source": "nvml"}
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        sm, smax, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in self.lines:
            f = [x.strip() for x in line.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                smax = float(f[2])
            except ValueError:
                continue
            for name, v in zip(names, f[5:9]):
                if v.lower() == "active":
                    reasons.add(name)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": smax,
                "reasons": sorted(reasons), "samples": len(sm), "source": "nvidia-smi"}


def workload_name(size):
    """The workload string both arms report (the same config: update + K + f_int of the J2 mesh
    in the same plastic state)."""
    return (f"J2 hex8 {size}^3 (sigma_y=200, E=200e3, nu=0.3, H=1e3), fused update+K+f_int, "
            f"plastic state")


def algorithmic_work(mesh_size, nnz, n_nodes, E, nqp, fp64=True):
    """Canonical algorithmic work of one J2 hex8 assembly (bytes, flops): K written once,
    connectivity, X, u, f_int, J2 state read (7 FP64) and written (7 FP64) per point; FLOPs
    29,040 per element (geometry, symmetric block B^T D B, f_int) + 250 per point (J2)."""
    kbytes = (8 if fp64 else 4) * nnz
    nbytes = 32 * E + 24 * n_nodes + 8 * 3 * n_nodes + 8 * 3 * n_nodes + 112 * nqp
    flops = (29040.0 + 8 * 250.0) * E
    return kbytes + nbytes, flops


def cpu_baseline_sample(threads=None, target_seconds=15.0):
    """The oracle (C++/OpenMP restatement of neon's path) timed on this host: update +
    assembly + internal force of a J2 hex8 mesh in the same plastic state, elements/s."""
    from oracle import binding as ob
    from neon_b200 import problem as P
    if threads:
        ob.set_threads(threads)
    cores = ob.max_threads()

    def run(n):
        pr = P.config_c3(n)
        om = ob.OracleMesh(pr.mesh.X, pr.mesh.conn, pr.material)
        u = plastic_displacement(pr.mesh)
        t0 = time.perf_counter()
        st, msg = om.update(u)
        om.assemble()
        om.internal_force()
        dt = time.perf_counter() - t0
        return pr.mesh.num_elements, dt

    E0, t0 = run(20)
    per_elem = t0 / E0
    n = 20
    for cand in (30, 40, 50, 60, 70, 80, 90, 100):
        if cand ** 3 * per_elem * 1.3 <= target_seconds:
            n = cand
    E, dt = run(n)
    reps = 1
    total = dt
    while total < target_seconds * 0.5 and reps < 5:
        _, d2 = run(n)
        total += d2
        reps += 1
    return {"value": E * reps / total, "unit": UNIT, "cores": cores, "kind": "port",
            "sample": f"oracle update+assembly+f_int of the J2 hex8 {n}^3 mesh ({E} elements, "
                      f"plastic state) x{reps}, {cores} OpenMP threads"}


def cpu_newton_baselines(args):
    """Newton-step wall times of the oracle (neon's CPU path restated: OpenMP assembly with
    binary-search atomics, RCM + Jacobi-PCG) on this host, all OpenMP threads: C1 in full, the
    first `cpu_c2_increments` increments of C2, the first increment of C3 (unless skipped) and
    the C3 PCG time per iteration on the assembled, Dirichlet-constrained first tangent."""
    from oracle import binding as ob
    from neon_b200 import problem as P
    out = {"cores": ob.max_threads(), "cpu": ob._cpu_model(), "kind": "port"}

    def solve(pr, label):
        t0 = time.perf_counter()
        rep, u, _, lg, _ = ob.static_solve(pr)
        dt = time.perf_counter() - t0
        nit = max(1, int(rep["newton_iterations"]))
        cg = int(lg[:, 2].sum()) if len(lg) else 0
        log(f"cpu {label}: {dt:.1f} s, {nit} Newton iterations, {cg} CG iterations")
        return {"status": int(rep["status"]), "seconds": dt, "load_steps": int(rep["load_steps"]),
                "newton_iterations": nit, "cg_iterations": cg, "newton_step_s": dt / nit}

    out["c1_full"] = solve(P.config_c1(20), "C1 20^3 full")
    pr = P.config_c2(64)
    pr.options.period = args.cpu_c2_increments * pr.options.initial
    out["c2"] = solve(pr, f"C2 64^3 {args.cpu_c2_increments} increment(s)")
    out["c2"]["increments"] = args.cpu_c2_increments
    if not args.cpu_skip_c3:
        pr = P.config_c3(100)
        pr.options.period = pr.options.initial
        out["c3_first_increment"] = solve(pr, "C3 100^3 first increment")
        # the PCG per iteration on the first tangent (a fixed count of iterations)
        om = ob.OracleMesh(pr.mesh.X, pr.mesh.conn, pr.material)
        om.update(np.zeros(om.ndofs))
        K = om.assemble()
        rp, col = om.pattern()
        its = 20
        secs, t_perm = ob.cg_sample_seconds(rp, col, K, np.ones(om.ndofs), its)
        out["c3_pcg"] = {"iterations_timed": its, "ms_per_iteration": 1e3 * secs / its,
                         "rcm_permutation_s": t_perm,
                         "note": "Jacobi-PCG iterations on P^T K P; the per-solve RCM "
                                 "permutation (rcm_permutation_s) is paid once per solve"}
    return out


def run_reference(args):
    """Reference arm: the reference's CPU algorithm (oracle port; the reference itself cannot be
    built here) on the same config, all host threads."""
    rank = _env_int("RANK", 0)
    if rank != 0:
        return 0
    from oracle import binding as ob
    from neon_b200 import problem as P
    cores = ob.max_threads()
    pr = P.config_c3(args.size)
    om = ob.OracleMesh(pr.mesh.X, pr.mesh.conn, pr.material)
    u = plastic_displacement(pr.mesh)
    E = pr.mesh.num_elements

    def step():
        om.save(False)  # revert to the committed (elastic) state: same return mapping each step
        om.update(u)
        om.assemble()
        om.internal_force()

    om.save(True)
    t0 = time.perf_counter()
    step()
    one = time.perf_counter() - t0
    # each step is bounded: keep the whole run within a few minutes
    budget = 150.0
    warm = max(0, min(args.warmup, int(budget / 4 / max(one, 1e-9))))
    steps = max(1, min(args.steps, int(budget / max(one, 1e-9))))
    for _ in range(warm):
        step()
    t0 = time.perf_counter()
    for _ in range(steps):
        step()
    dt = time.perf_counter() - t0
    value = E * steps / dt
    line = {"metric": METRIC, "value": value, "unit": UNIT, "impl": "reference", "n_gpus": 1,
            "steps": steps, "warmup": warm, "ms_per_step": 1e3 * dt / steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic",
            "config": {"workload": workload_name(args.size),
                       "elements": E, "dofs": om.ndofs, "nnz": int(om.nnz),
                       "parallelism": "replicas x1",
                       "l2": "inputs larger than L2 (K 1.96 GB, state 0.45 GB)"},
            "cpu_baseline": {"value": value, "unit": UNIT, "cores": cores, "kind": "port",
                             "sample": f"{steps} full assemblies of the {args.size}^3 mesh on "
                                       f"{cores} OpenMP threads"},
            "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--size", type=int, default=100)
    ap.add_argument("--newton-load-steps", type=int, default=2)
    ap.add_argument("--newton-cyclic-increments", type=int, default=24,
                    help="increments of the cyclic segment (80 = the whole 20-step cycle)")
    ap.add_argument("--newton-cyclic-sensitivity", action="store_true",
                    help="also run the cyclic segment in FP64 at rtol 1e-11")
    ap.add_argument("--no-newton", action="store_true")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--e2e-steps", type=int, default=3)
    ap.add_argument("--cg-iterations", type=int, default=200)
    ap.add_argument("--batch-instances", type=int, default=256)
    ap.add_argument("--no-batch", action="store_true")
    ap.add_argument("--batch-delta", type=float, default=1e-2,
                    help="reliable-update interval of the batched mixed path")
    ap.add_argument("--no-adjoint", action="store_true")
    ap.add_argument("--no-c2", action="store_true")
    ap.add_argument("--adjoint-size", type=int, default=48)
    ap.add_argument("--cpu-newton", action="store_true",
                    help="only time the oracle's Newton steps (C1, C2, C3) and print them")
    ap.add_argument("--cpu-c2-increments", type=int, default=1)
    ap.add_argument("--cpu-skip-c3", action="store_true")
    args = ap.parse_args()
    if args.cpu_newton:
        print(json.dumps({"cpu_newton": cpu_newton_baselines(args)}), flush=True)
        return 0
    if args.impl == "reference":
        return run_reference(args)

    import torch
    rank, world, local = _env_int("RANK", 0), _env_int("WORLD_SIZE", 1), _env_int("LOCAL_RANK", 0)
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600),
                                device_id=torch.device("cuda", local))
    from neon_b200 import api, build
    from neon_b200 import problem as P
    build.build()
    warmup = max(3, args.warmup)

    pr = P.config_c3(args.size)
    mesh = api.SolidMesh(pr.mesh.X, pr.mesh.conn, pr.material)
    stream = torch.cuda.Stream()
    mesh.set_stream(stream.cuda_stream)
    E, nqp = pr.mesh.num_elements, mesh.nqp
    u = plastic_displacement(pr.mesh)
    mesh.save_internal_variables(True)  # committed state: zero plastic strain
    mesh.set_displacement(u)

    def assembly_step():
        mesh.save_internal_variables(False)  # revert: every step runs the same return mapping
        ev0.record(stream)
        mesh.update_assemble_device(api.FP64)
        ev1.record(stream)

    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    for _ in range(warmup):
        assembly_step()
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    clocks = ClockSampler(local)
    clocks.start()
    torch.cuda.synchronize()
    launches0 = mesh.launches()
    kernel_ms = []
    tw0 = torch.cuda.Event(enable_timing=True)
    tw1 = torch.cuda.Event(enable_timing=True)
    tw0.record(stream)
    for _ in range(args.steps):
        assembly_step()
        ev1.synchronize()
        kernel_ms.append(ev0.elapsed_time(ev1))
    tw1.record(stream)
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    launches = mesh.launches() - launches0
    region_ms = tw0.elapsed_time(tw1)
    clock_info = clocks.stop()
    t_asm = sum(kernel_ms) / len(kernel_ms) * 1e-3
    t_max = t_asm
    if dist:
        t_max = max_over_ranks(t_asm, dist)
    value = world * E / t_max
    # the same assembly with the colour-partitioned, bit-reproducible scatter (the Newton
    # driver's mode), outside the headline's timed region
    mesh.set_scatter_mode(api.SCATTER_COLOURED)
    for _ in range(warmup):
        assembly_step()
    col_ms = []
    for _ in range(args.steps):
        assembly_step()
        ev1.synchronize()
        col_ms.append(ev0.elapsed_time(ev1))
    mesh.set_scatter_mode(api.SCATTER_RED)
    coloured = {"ms_per_step": sum(col_ms) / len(col_ms),
                "elements_per_s": E / (sum(col_ms) / len(col_ms) * 1e-3),
                "note": "K and f_int zeroed, then one launch per element colour adding into them "
                        "(no entry gets two additions in one launch, so every sum runs in colour "
                        "order): bit-reproducible K and f_int (nb2_static_solve always uses it)"}

    # roofline of the dominant kernel (the fused element kernel)
    peaks = {}
    try:
        peaks = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))
    except (OSError, ValueError):
        pass
    hbm = float(peaks.get("hbm_gbs", 6650.0))
    hbm_src = "measured" if "hbm_gbs" in peaks else "fallback"
    fp64_peak = api.probe_fma_throughput(True)
    fp32_peak = api.probe_fma_throughput(False)
    alg_bytes, alg_flops = algorithmic_work(args.size, mesh.nnz, pr.mesh.num_nodes, E, nqp)
    t_hbm = alg_bytes / (hbm * 1e9)
    t_fp = alg_flops / fp64_peak
    traffic = None
    tfile = os.path.join(ROOT, "profiles", "traffic.json")
    if os.path.exists(tfile):
        try:
            traffic = json.load(open(tfile)).get("k_element_fp64_j2_hex8_bytes_per_launch")
        except (OSError, ValueError):
            traffic = None
    if t_fp >= t_hbm:
        roof = {"bound": "fp64", "achieved": alg_flops / t_asm / 1e12,
                "peak": fp64_peak / 1e12, "unit": "TFLOP/s",
                "frac": (alg_flops / t_asm) / fp64_peak, "traffic": traffic,
                "peak_source": "measured (FP64 FMA-chain probe, this run)",
                "hbm": {"achieved": alg_bytes / t_asm / 1e9, "peak": hbm, "unit": "GB/s",
                        "frac": (alg_bytes / t_asm / 1e9) / hbm, "peak_source": hbm_src},
                "algorithmic_bytes": alg_bytes, "algorithmic_flops": alg_flops}
    else:
        roof = {"bound": "hbm", "achieved": alg_bytes / t_asm / 1e9, "peak": hbm, "unit": "GB/s",
                "frac": (alg_bytes / t_asm / 1e9) / hbm, "traffic": traffic,
                "peak_source": hbm_src, "algorithmic_bytes": alg_bytes,
                "algorithmic_flops": alg_flops}

    log(f"assembly: {t_asm * 1e3:.3f} ms")
    pcg = None
    if args.cg_iterations > 0:
        pcg = pcg_timing(api, torch, stream, mesh, pr, args.cg_iterations, hbm)

    log("pcg timing done")
    e2e = None
    if not args.no_e2e:
        e2e = end_to_end(api, args, pr, u, world, dist, torch, E)

    log("e2e done")
    newton = None
    if not args.no_newton:
        newton = newton_comparison(api, P, args, mesh)

    log("newton done")
    c2 = c1 = None
    if not args.no_newton and not args.no_c2:
        c2 = c2_newton(api, P)
        c1 = c2_newton(api, P, "c1")
    adjoint = None
    if not args.no_adjoint:
        adjoint = adjoint_timing(api, P, args)
    batched = None
    if not args.no_batch and args.batch_instances > 0:
        batched = batched_comparison(api, P, args)

    log("batched done")
    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu:
        cpu = cpu_baseline_sample()

    line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": warmup, "ms_per_step": t_max * 1e3, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": workload_name(args.size),
                       "elements": E, "dofs": mesh.ndofs, "nnz": mesh.nnz,
                       "parallelism": f"replicas x{world}",
                       "l2": "inputs larger than L2 (K 1.96 GB, state 0.45 GB)"},
            "scatter": "red.global.add into zeroed K and f_int (NB2_SCATTER_RED, the default "
                       "for standalone assembly)",
            "coloured_scatter": coloured, "roofline": roof, "cpu_baseline": cpu, "e2e": e2e, "gpu_launches": int(launches),
            "timed_region_ms": region_ms, "clocks": clock_info,
            "fp32_fma_peak_tflops": fp32_peak / 1e12, "pcg": pcg, "newton": newton,
            "c1_newton": c1, "c2_newton": c2, "adjoint": adjoint, "batched": batched}
    if rank == 0:
        print(json.dumps(line), flush=True)
    mesh.close()
    if dist:
        dist.barrier()
        dist.destroy_process_group()
    return 0


def pcg_timing(api, torch, stream, mesh, pr, iters, hbm):
    """Per-iteration device time of the PCG on the full K (FP64 and FP32), and its bandwidth
    against the algorithmic bytes of one iteration."""
    dofs = np.concatenate([t.dofs for t in pr.dirichlet if t.name == "bottom"])
    mesh.set_dirichlet_mask(dofs)
    n, nnz, nnzb, N = mesh.ndofs, mesh.nnz, mesh.nnzb, pr.mesh.num_nodes
    out = {}
    for name, prec in (("fp64", api.FP64), ("fp32", api.MIXED)):
        if prec == api.MIXED:
            mesh.save_internal_variables(False)
            mesh.update_assemble_device(api.MIXED)
        sv = 8 if prec == api.FP64 else 4
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        times = {}
        for its in (20, iters + 20):
            mesh.solve_device(prec, 0.0, its)  # warm (graph capture on first use)
            e0.record(stream)
            mesh.solve_device(prec, 0.0, its)
            e1.record(stream)
            torch.cuda.synchronize()
            times[its] = e0.elapsed_time(e1)
        ms = (times[iters + 20] - times[20]) / iters
        # matrix values + block columns + block row pointers, 13 vector streams, Dirichlet mask
        alg = sv * nnz + 4 * nnzb + 4 * (N + 1) + 13 * sv * n + n
        out[name] = {"ms_per_iteration": ms, "algorithmic_bytes": alg,
                     "achieved_gbs": alg / (ms * 1e-3) / 1e9,
                     "frac_of_hbm": alg / (ms * 1e-3) / 1e9 / hbm}
    out["fp32_over_fp64_speedup"] = out["fp64"]["ms_per_iteration"] / out["fp32"]["ms_per_iteration"]
    return out


def end_to_end(api, args, pr, u, world, dist, torch, E):
    """The metric through the drop-in C-ABI with host buffers, copies inside the timed region."""
    mesh_e2e = api.SolidMesh(pr.mesh.X, pr.mesh.conn, pr.material)
    mesh_e2e.save_internal_variables(True)
    # page-locked host buffers (a caller pins its K value array once, e.g. cudaHostRegister)
    Kh = torch.zeros(mesh_e2e.nnz, dtype=torch.float64, pin_memory=True).numpy()
    fh = torch.zeros(mesh_e2e.ndofs, dtype=torch.float64, pin_memory=True).numpy()
    uh = torch.zeros(mesh_e2e.ndofs, dtype=torch.float64, pin_memory=True).numpy()
    uh[:] = u
    L = api.lib()

    def e2e_step():
        mesh_e2e.save_internal_variables(False)
        api._check(L.nb2_update_internal_variables(mesh_e2e.h, uh.ctypes.data, 0.0), mesh_e2e.h)
        api._check(L.nb2_assemble(mesh_e2e.h, Kh.ctypes.data, fh.ctypes.data), mesh_e2e.h)

    e2e_step()
    t0 = time.perf_counter()
    for _ in range(args.e2e_steps):
        e2e_step()
    t_e2e = (time.perf_counter() - t0) / args.e2e_steps
    if dist:
        t_e2e = max_over_ranks(t_e2e, dist)
    e2e = {"value": world * E / t_e2e, "unit": UNIT, "h2d_bytes_per_step": 8 * mesh_e2e.ndofs,
           "d2h_bytes_per_step": 8 * mesh_e2e.nnz + 8 * mesh_e2e.ndofs,
           "call": "nb2_update_internal_variables + nb2_assemble (host u in, host CSR K + f_int "
                   "out; page-locked host buffers)"}
    mesh_e2e.close()
    return e2e


def _newton_run(api, P, n, steps, prec, delta=None, cg_tol=None):
    pr = P.config_c3(n)
    pr.options.period = float(steps) * pr.options.initial
    if cg_tol is not None:
        pr.options.cg_tolerance = cg_tol
    sm = api.StaticMatrix(pr, precision=prec,
                          mixed_inner_tolerance=MIXED_DELTA if delta is None else delta)
    try:
        u = sm.solve(raise_on_error=False)
    finally:
        sm.mesh.close()
    r = sm.report
    nit = max(1, int(r["newton_iterations"]))
    return u, {"status": int(r["status"]), "load_steps": int(r["load_steps"]),
               "newton_iterations": int(r["newton_iterations"]),
               "cg_iterations": int(r["cg_iterations"]), "seconds_total": r["seconds_total"],
               "newton_step_s": r["seconds_total"] / nit,
               "device_s_elements": r["seconds_update_assembly"],
               "device_s_solve": r["seconds_solve"],
               "ms_per_cg_iteration": 1e3 * r["seconds_solve"] / max(1, int(r["cg_iterations"]))}


def _rel(a, b):
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


def newton_comparison(api, P, args, mesh_unused):
    """FP64 vs mixed device Newton on the 100^3 J2 mesh, Newton-step seconds = the segment's
    wall time over its Newton iterations (update, assembly or stored tangent, Dirichlet, PCG to
    rtol 1e-10, norms):
      first_increment  the first load increment (elastic range);
      yielding         the first `newton_load_steps` increments (points yield);
      cyclic           the first `newton_cyclic_increments` increments of the 80-increment
                       cycle (24 = t in [0, 6]: past the load reversal at t = 5, where the top
                       face starts to unload); 80 runs the whole cycle.  Increments that do not
                       converge are halved (neon's adaptive stepping), so the segment's Newton
                       iterations include those of the failed attempts; `completed` says both
                       paths reached the segment's end time.
    The reference's J2 update mutates the plastic strain at every Newton iteration, so once
    points yield the converged displacement depends on the Newton path.  The FP64 path is bit
    reproducible (fixed-order assembly and reductions): `fp64_rerun_rel_err_u` is that check;
    `fp64_rtol_sensitivity_rel_err_u` (rtol 1e-10 vs 1e-11) measures how far a perturbation of
    the iterates at the CG tolerance moves the converged displacement, the scale any other
    solver meets; the mixed path is also compared at rtol 1e-12 on both paths."""
    delta = MIXED_DELTA
    out = {"mixed_method": "reliable-update PCG: FP32 matrix-free tangent, FP64 residual "
                           f"replacement every {delta:g} reduction, same rtol as FP64",
           "segments": {}}
    segs = [("first_increment", 1), ("yielding", args.newton_load_steps)]
    if args.newton_cyclic_increments > 0:
        segs.append(("cyclic", args.newton_cyclic_increments))
    for name, steps in segs:
        u64, r64 = _newton_run(api, P, args.size, steps, api.FP64)
        log(f"newton {name} fp64: {r64['seconds_total']:.2f} s")
        u32, r32 = _newton_run(api, P, args.size, steps, api.MIXED, delta)
        log(f"newton {name} mixed: {r32['seconds_total']:.2f} s")
        seg = {"load_steps_run": steps, "fp64": r64, "mixed": r32,
               "completed": r64["status"] == 0 and r32["status"] == 0,
               "mixed_rel_err_u": _rel(u32, u64),
               "newton_step_speedup": r64["newton_step_s"] / max(r32["newton_step_s"], 1e-12),
               "solve_speedup": r64["seconds_total"] / max(r32["seconds_total"], 1e-12)}
        if name == "yielding":
            u64r, _ = _newton_run(api, P, args.size, steps, api.FP64)
            seg["fp64_rerun_rel_err_u"] = _rel(u64r, u64)
            seg["fp64_rerun_bitwise_equal"] = bool(np.array_equal(u64r, u64))
            u64b, _ = _newton_run(api, P, args.size, steps, api.FP64, cg_tol=1e-11)
            seg["fp64_rtol_sensitivity_rel_err_u"] = _rel(u64b, u64)
            # both paths at a tighter CG tolerance
            t64, q64 = _newton_run(api, P, args.size, steps, api.FP64, cg_tol=1e-12)
            t32, q32 = _newton_run(api, P, args.size, steps, api.MIXED, delta, cg_tol=1e-12)
            seg["rtol_1e-12"] = {
                "fp64": q64, "mixed": q32, "mixed_rel_err_u": _rel(t32, t64),
                "newton_step_speedup": q64["newton_step_s"] / max(q32["newton_step_s"], 1e-12)}
            log(f"newton {name} rtol 1e-12: mixed err {seg['rtol_1e-12']['mixed_rel_err_u']:.2e}")
        if name == "cyclic" and args.newton_cyclic_sensitivity:
            # the FP64 path against itself at rtol 1e-11 over the same cycle segment
            u64b, _ = _newton_run(api, P, args.size, steps, api.FP64, cg_tol=1e-11)
            seg["fp64_rtol_sensitivity_rel_err_u"] = _rel(u64b, u64)
            log(f"newton {name} fp64 rtol sensitivity {seg['fp64_rtol_sensitivity_rel_err_u']:.2e}")
        out["segments"][name] = seg
    main = out["segments"]["cyclic" if "cyclic" in out["segments"] else "yielding"]
    out["newton_step_s_fp64"] = main["fp64"]["newton_step_s"]
    out["newton_step_s_mixed"] = main["mixed"]["newton_step_s"]
    out["newton_step_speedup"] = main["newton_step_speedup"]
    out["mixed_rel_err_u"] = main["mixed_rel_err_u"]
    return out


def c2_newton(api, P, config="c2"):
    """Config 2 in full (neo-Hooke, jittered 64^3 hex8, 823,875 DOFs, stretch to 1.3 in 10
    increments), or config 1 in full (linear elasticity, 20^3, one increment): FP64 and mixed
    device Newton, seconds per Newton step and the relative difference of the final
    displacements (neither model is path dependent)."""
    out = {}
    us = {}
    for name, prec in (("fp64", api.FP64), ("mixed", api.MIXED)):
        pr = P.config_c2(64) if config == "c2" else P.config_c1(20)
        sm = api.StaticMatrix(pr, precision=prec, mixed_inner_tolerance=MIXED_DELTA)
        try:
            us[name] = sm.solve(raise_on_error=False)
        finally:
            sm.mesh.close()
        r = sm.report
        nit = max(1, int(r["newton_iterations"]))
        out[name] = {"status": int(r["status"]), "load_steps": int(r["load_steps"]),
                     "newton_iterations": nit, "cg_iterations": int(r["cg_iterations"]),
                     "seconds_total": r["seconds_total"], "newton_step_s": r["seconds_total"] / nit}
        log(f"{config} {name}: {r['seconds_total']:.2f} s")
    out["mixed_rel_err_u"] = _rel(us["mixed"], us["fp64"])
    out["newton_step_speedup"] = out["fp64"]["newton_step_s"] / max(out["mixed"]["newton_step_s"],
                                                                   1e-12)
    return out


def adjoint_timing(api, P, args):
    """Config 4 at 48^3: the forward solve and the adjoint gradient dJ/dG_e of
    J = 1/2 |u_top - u_target|^2 over all 110,592 per-element shear moduli, FP64 and with the
    FP32-bulk inner solves; seconds of each and the relative difference of the two gradients.
    The central-difference check of the gradient is in tests/test_gpu_adjoint.py."""
    n = args.adjoint_size
    target = P.config_c4(n, seed_field=99)
    sm_t = api.StaticMatrix(target)
    u_target = sm_t.solve()
    sm_t.mesh.close()
    pr = P.config_c4(n, seed_field=7)
    sm = api.StaticMatrix(pr)
    t0 = time.perf_counter()
    u = sm.solve()
    t_fwd = time.perf_counter() - t0
    top = np.unique(pr.mesh.faces["top"].reshape(-1))
    dofs = (3 * top[:, None] + np.arange(3)).reshape(-1)
    g = np.zeros_like(u)
    g[dofs] = u[dofs] - u_target[dofs]
    out = {"mesh": f"{n}^3 hex8 ({pr.mesh.num_elements} elements, {3 * pr.mesh.num_nodes} DOFs)",
           "forward_solve_s": t_fwd, "forward_newton_iterations":
           int(sm.report["newton_iterations"])}
    grads = {}
    for name, prec in (("fp64", api.FP64), ("mixed", api.MIXED)):
        sm.mesh.adjoint_shear_gradient(g, prec, 1e-10)  # warm (buffers, graphs)
        t0 = time.perf_counter()
        grads[name] = sm.mesh.adjoint_shear_gradient(g, prec, 1e-10)
        dt = time.perf_counter() - t0
        out[name] = {"adjoint_s": dt, "inner_iterations": int(sm.mesh.adjoint_iterations)}
        log(f"adjoint {name}: {dt * 1e3:.1f} ms")
    out["mixed_vs_fp64_rel_err_grad"] = _rel(grads["mixed"], grads["fp64"])
    out["adjoint_over_forward"] = out["fp64"]["adjoint_s"] / max(t_fwd, 1e-12)
    sm.mesh.close()
    return out


def batched_comparison(api, P, args):
    """The batched workload: config_c5 instances (tet4 boxes of uneven size, neo-Hooke with
    per-instance mu) solved in one context, FP64 and mixed; one instance cross-checked against
    its own single solve."""
    sizes = P.config_c5_sizes(args.batch_instances)
    probs = [P.config_c5_instance(m, mu) for m, mu in sizes]
    out = {"instances": len(probs),
           "dofs": int(sum(3 * p.mesh.num_nodes for p in probs)),
           "elements": int(sum(p.mesh.num_elements for p in probs))}
    sols = {}
    for name, prec in (("fp64", api.FP64), ("mixed", api.MIXED)):
        bs = api.BatchedStaticMatrix(probs, precision=prec,
                                     mixed_inner_tolerance=args.batch_delta)
        t0 = time.perf_counter()
        u = bs.solve(raise_on_error=False)
        dt = time.perf_counter() - t0
        log(f"batched {name}: {dt:.2f} s")
        reps = bs.reports
        out[name] = {"seconds": dt, "instances_per_s": len(probs) / dt,
                     "ok": int(sum(r["status"] == 0 for r in reps)),
                     "newton_iterations_max": int(max(r["newton_iterations"] for r in reps)),
                     "cg_iterations_max": int(max(r["cg_iterations"] for r in reps)),
                     "device_s_elements": reps[0]["seconds_update_assembly"],
                     "device_s_solve": reps[0]["seconds_solve"], "tuned": bs.tuned}
        sols[name] = (u, bs.node_offsets)
        bs.mesh.close()
    (u64, off), (u32, _) = sols["fp64"], sols["mixed"]
    errs = [_rel(u32[3 * off[i]:3 * off[i + 1]], u64[3 * off[i]:3 * off[i + 1]])
            for i in range(len(probs))]
    out["mixed_rel_err_u_max"] = float(max(errs))
    out["speedup_mixed"] = out["fp64"]["seconds"] / max(out["mixed"]["seconds"], 1e-12)
    k = int(np.argmax([m for m, _ in sizes]))
    sm = api.StaticMatrix(probs[k])
    try:
        us = sm.solve(raise_on_error=False)
    finally:
        sm.mesh.close()
    out["largest_instance_vs_single_rel_err_u"] = _rel(u64[3 * off[k]:3 * off[k + 1]], us)
    return out


if __name__ == "__main__":
    sys.exit(main())
