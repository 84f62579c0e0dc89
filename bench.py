"""Benchmark: GDoF/s of the Euler operator explicit apply (fused stage-1 right-hand side
triple: density, velocity, pressure) on the 2D terrain-following 512x256 mesh, degree 4, FP64.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference] [--no-sweep] [--no-solvers]

One step = one fused apply over the whole mesh with inputs resident in HBM (`value`);
`e2e` is the same apply through the host-buffer C-ABI call (pinned host inputs copied in,
all four outputs copied back, every step).  The inputs (7 scalar FP64 fields, 183 MB) and
outputs (105 MB) exceed the 126 MB L2, so no L2 flush is needed between steps.
N > 1: one process per GPU (torchrun), independent replicas ("replicas only": the
operator apply has no cross-GPU exchange in this library), max time over ranks.
--impl reference: the tuned CPU port of the same apply (oracle/af_cpu_port.cpp, checked against
the CPU oracle; the reference itself needs deal.II, which is not installable here) on all host
cores, on the same 512x32 strip as the cpu_baseline leg, same metric.
Rank 0 also reports the second half of the metric (`imex`: s per IMEX step, FP64 vs mixed
precision at the same solver tolerance) and the Schur pressure solve (`schur_solve`).
"""
import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

NX, NZ, DEGREE, STAGE = 512, 256, 4, 1
SEED = 20261203
METRIC = "GDoF/s per Euler operator apply"
PROFILE = os.path.join(ROOT, "profiles", "rhs_fused_stage1_p4_512x256.md")


def workload(P=DEGREE, nx=NX, nz=NZ, modes=16):
    """Stage-1 sources: rho0, u0, p0 from the seeded 16x16-mode state; rho_tmp_2 and
    u_fixed from an independent 4x4-mode state (distinct arrays, so nothing aliases)."""
    from atmospheric_flows_b200 import mesh as M
    m = M.hill_mesh(nx, nz)
    st = M.hill_state(m, P, seed=SEED, modes=modes)
    st2 = M.hill_state(m, P, seed=SEED + 1, modes=4)
    src = [st.rho, st.u, st.p, st2.rho, st2.u]
    return m, src


def config(P=DEGREE):
    nd = NX * NZ * (P + 1) ** 2
    return {
        "workload": f"EulerOperator explicit apply: stage-1 rhs triple (density+velocity+pressure, one fused "
                    f"launch) on the 2D terrain-following hill mesh {NX}x{NZ}, degree {P}, QGauss({2 * P + 1}), FP64",
        "mesh": f"{NX}x{NZ} cells, Witch of Agnesi h0=400 m a=1 km, x in [-20,20] km, top 16 km, walls",
        "degree": P, "dofs_per_apply": 4 * nd,
        "inputs": "rho0, u0 (2), p0, rho_tmp_2, u_fixed (2): 7 scalar fields, 183 MB > L2 (no flush needed)",
        "state": f"hydrostatic background (theta0=300 K, N=0.01/s) + 16x16-mode Fourier perturbation 1e-3, seed {SEED}",
        "parallelism": "replicas",
    }


def measured_peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(path):
        with open(path) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def profile_numbers():
    """traffic / executed FP64 flops per launch from the committed ncu summary."""
    out = {}
    if os.path.exists(PROFILE):
        for line in open(PROFILE):
            for key in ("traffic_bytes_per_launch", "fp64_flops_per_launch"):
                if line.strip().startswith(key + ":"):
                    out[key] = float(line.split(":", 1)[1].strip().split()[0])
    return out


def gpu_pci_id(dev):
    """The PCI bus id of a torch CUDA device in NVML's and nvidia-smi's form, or None."""
    try:
        import torch
        pr = torch.cuda.get_device_properties(dev)
        return f"{pr.pci_domain_id:08x}:{pr.pci_bus_id:02x}:{pr.pci_device_id:02x}.0"
    except Exception:
        return None


_REASONS = (("hw_slowdown", 0x8), ("hw_thermal_slowdown", 0x40), ("sw_thermal_slowdown", 0x20),
            ("sw_power_cap", 0x4))


class Clocks:
    """SM clocks and throttle reasons around the timed region: nvidia-smi every 100 ms with
    timestamps, and NVML read every 2 ms by a thread (the timed region of a short run is a few
    ms).  mark() the region's start and end; the summary keeps the samples inside it (NVML's
    when there are any, else nvidia-smi's, else all samples, flagged).  `gpu` is the device's
    PCI bus id (or an index); `nvml` a module with pynvml's interface (tests pass a fake)."""

    def __init__(self, gpu, nvml=None):
        self.gpu = gpu
        self.f = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
        self.p = None
        self.t0 = self.t1 = None
        self.nv_rows = []
        self._nv = nvml
        self._stop = None
        self._thread = None

    def _nvml_handle(self):
        nv = self._nv
        if nv is None:
            import pynvml as nv
            self._nv = nv
        nv.nvmlInit()
        if isinstance(self.gpu, str):
            return nv.nvmlDeviceGetHandleByPciBusId(self.gpu)
        return nv.nvmlDeviceGetHandleByIndex(int(self.gpu))

    def _poll(self, h):
        nv = self._nv
        mx = nv.nvmlDeviceGetMaxClockInfo(h, nv.NVML_CLOCK_SM)
        while not self._stop.is_set():
            try:
                sm = nv.nvmlDeviceGetClockInfo(h, nv.NVML_CLOCK_SM)
                bits = nv.nvmlDeviceGetCurrentClocksEventReasons(h)
            except Exception:
                break
            self.nv_rows.append((time.time(), float(sm), float(mx), {n for n, b in _REASONS if bits & b}))
            self._stop.wait(0.002)

    def __enter__(self):
        import threading
        q = ("timestamp,index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
        try:
            self.p = subprocess.Popen(["nvidia-smi", f"--id={self.gpu}", f"--query-gpu={q}", "--format=csv,noheader,nounits",
                                       "-lms", "100"], stdout=self.f, stderr=subprocess.DEVNULL)
        except (FileNotFoundError, OSError):
            self.p = None
        try:
            h = self._nvml_handle()
            self._stop = threading.Event()
            self._thread = threading.Thread(target=self._poll, args=(h,), daemon=True)
            self._thread.start()
        except Exception:
            self._thread = None
        time.sleep(0.3)
        return self

    def mark(self):
        """Call at the start and at the end of the timed region (after a device sync)."""
        if self.t0 is None:
            self.t0 = time.time()
        else:
            self.t1 = time.time()

    def __exit__(self, *a):
        if self.p:
            time.sleep(0.15)  # one more sample after the region
            self.p.terminate()
            self.p.wait()
        if self._thread:
            self._stop.set()
            self._thread.join()

    def summary(self):
        import datetime
        inside = lambda rows: [r for r in rows if self.t0 is not None and self.t1 is not None and
                               self.t0 <= r[0] <= self.t1]
        nv_in = inside(self.nv_rows)
        if nv_in:
            use, window = nv_in, "timed region (NVML every 2 ms)"
        else:
            self.f.flush()
            self.f.seek(0)
            rows = []
            names = [n for n, _ in _REASONS]
            for line in self.f:
                parts = [x.strip() for x in line.split(",")]
                if len(parts) < 10:
                    continue
                try:
                    ts = datetime.datetime.strptime(parts[0], "%Y/%m/%d %H:%M:%S.%f").timestamp()
                    rows.append((ts, float(parts[2]), float(parts[3]),
                                 {n for n, v in zip(names, parts[6:10]) if v.lower() == "active"}))
                except ValueError:
                    continue
            smi_in = inside(rows)
            use = smi_in or rows
            window = "timed region" if smi_in else "around the timed region (shorter than the sampling interval)"
        sm = [r[1] for r in use]
        reasons = set().union(*(r[3] for r in use)) if use else set()
        return {"sm_mhz": statistics.median(sm) if sm else None,
                "sm_max_mhz": max((r[2] for r in use), default=None),
                "reasons": sorted(reasons), "samples": len(sm), "window": window}


CPU_ROWS = 32  # the CPU sample: a 512x32 strip of the workload mesh, 1/8 of its cells


def cpu_sample(rows=CPU_ROWS):
    """The strip both CPU measurements and the parity check run on: the bottom `rows` rows of
    the hill domain (same x extent and cell width, top at 16 km * rows / 256), the workload's
    state construction."""
    from atmospheric_flows_b200 import mesh as M
    m = M.hill_mesh(NX, rows, top=16000.0 * rows / NZ)
    st = M.hill_state(m, DEGREE, seed=SEED)
    st2 = M.hill_state(m, DEGREE, seed=SEED + 1, modes=4)
    return m, [st.rho, st.u, st.p, st2.rho, st2.u]


def cpu_sample_label(rows=CPU_ROWS):
    return (f"{NX}x{rows} strip of the {NX}x{NZ} workload mesh (1/{NZ // rows} of its cells) per step, the same "
            f"strip in the reference arm and in the cpu_baseline leg")


def time_cpu_port(m, src, warmup, steps, threads):
    """Mean seconds per fused stage-1 apply of the tuned CPU port (oracle/af_cpu_port.cpp:
    sum factorisation vectorised over cells, each face once, OpenMP) on the host cores."""
    from oracle.oracle import cpu_port_rhs_fused_stage1, set_num_threads
    from atmospheric_flows_b200 import mesh as M
    set_num_threads(threads)
    sc = M.Scaling()
    f = lambda: cpu_port_rhs_fused_stage1(m, DEGREE, sc.Ma, sc.Fr, 2.0, src)
    for _ in range(max(1, warmup)):
        f()
    t = time.perf_counter()
    for _ in range(steps):
        f()
    return (time.perf_counter() - t) / steps


CPU_NOTE = ("tuned CPU port of the fused stage-1 rhs (oracle/af_cpu_port.cpp: sum factorisation vectorised over "
            "batches of 4 cells, each face once, OpenMP; checked against the oracle at 1e-12); the reference "
            "itself needs deal.II >= 9.3 + MPI + p4est, unavailable here")


def run_reference(args, rank):
    if rank != 0:
        return
    threads = os.cpu_count() or 1
    m, src = cpu_sample()
    dt = time_cpu_port(m, src, args.warmup, args.steps, threads)
    dofs = 4 * m.n_cells * (DEGREE + 1) ** 2
    v = dofs / dt / 1e9
    line = {"metric": METRIC, "value": v, "unit": "GDoF/s", "impl": "reference", "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": dt * 1e3, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic", "config": config(),
            "cpu_baseline": {"value": v, "unit": "GDoF/s", "cores": threads, "kind": "port",
                             "sample": cpu_sample_label(), "note": CPU_NOTE},
            "e2e": {"value": v, "unit": "GDoF/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def strip_parity(dev, stream):
    """GPU fused apply vs the oracle on the identical CPU-sample strip: the largest relative L2
    difference over the density, velocity and pressure outputs."""
    import torch
    from atmospheric_flows_b200 import mesh as M
    from atmospheric_flows_b200.operator import EULEROperator
    from oracle.oracle import OracleOperator
    m, src = cpu_sample()
    sc = M.Scaling()
    ns = m.n_cells * (DEGREE + 1) ** 2
    op = EULEROperator(m, DEGREE, sc.Ma, sc.Fr, 2.0, stream=stream)
    op.set_HYPERBOLIC_stage(STAGE)
    out = [torch.empty(k * ns, dtype=torch.float64, device=dev) for k in (1, 2, 1)]
    op.vmult_rhs_fused(*out, [torch.from_numpy(a).to(dev) for a in src])
    stream.synchronize()
    o = OracleOperator(m, DEGREE, sc.Ma, sc.Fr, 2.0)
    o.set_HYPERBOLIC_stage(STAGE)
    want = [o.vmult_rhs_rho_update(src[:2]), o.vmult_rhs_velocity_fixed(src[:4]), o.vmult_rhs_pressure(src)]
    return max(float(np.linalg.norm(g.cpu().numpy() - w) / np.linalg.norm(w)) for g, w in zip(out, want))


def time_device(op, bufs, src, stream, K, W):
    import torch
    for _ in range(W):
        op.vmult_rhs_fused(*bufs, src)
    stream.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(K):
        op.vmult_rhs_fused(*bufs, src)
    e1.record(stream)
    e1.synchronize()
    return e0.elapsed_time(e1) * 1e-3 / K


def run_solvers(dev):
    """The second half of the metric, s per IMEX step FP64 vs mixed at the same tolerance, and
    the Schur pressure solve those steps are made of (device time, CUDA events)."""
    import torch
    from atmospheric_flows_b200 import mesh as M
    from atmospheric_flows_b200.imex import IMEXStepper
    from atmospheric_flows_b200.operator import EULEROperator
    from atmospheric_flows_b200.schur import SchurSolver
    sc = M.Scaling()
    P = DEGREE
    d = lambda a: torch.from_numpy(np.ascontiguousarray(a)).to(dev)
    out = {}
    # ---- Schur pressure solve: 1024x256 hill mesh, degree 4, seeded smooth rhs, rel. residual 1e-10
    nx, nz, dt = 1024, 256, 0.5
    m = M.hill_mesh(nx, nz)
    st = M.hill_state(m, P, seed=SEED, modes=4)
    rhs = M.hill_state(m, P, seed=SEED + 7, modes=8, amplitude=1e-2).p - 1.0
    op = EULEROperator(m, P, sc.Ma, sc.Fr, dt)
    op.set_stream(torch.cuda.current_stream(dev))
    op.set_schur_mode(1)
    op.set_HYPERBOLIC_stage(1)
    op.set_rho_for_fixed(d(st.rho))
    op.set_pres_fixed(d(st.p))
    b = d(rhs)
    sol = {}
    res = {}
    for pc in ("jacobi", "mg_fp64", "mg_fp32", "cheb_fp64", "cheb_fp32"):
        s = SchurSolver(op, pc)
        torch.cuda.synchronize(dev)
        t = time.perf_counter()
        s.setup()
        torch.cuda.synchronize(dev)
        t_setup = time.perf_counter() - t
        for _ in range(2):  # the second solve is timed (first includes lazy allocations)
            x = torch.zeros_like(b)
            r = s.solve(x, b, rel_tol=1e-10, max_iterations=5000)
        sol[pc] = x
        res[pc] = {"iterations": r["iterations"], "solve_s": r["seconds"], "setup_s": t_setup,
                   "levels": len(s.levels())}
        del s
    for pc in res:
        res[pc]["rel_error_vs_fp64_jacobi"] = float(torch.linalg.norm(sol[pc] - sol["jacobi"]) /
                                                    torch.linalg.norm(sol["jacobi"]))
    out["schur_solve"] = {
        "config": f"(D - C A^-1 B) p = b on the hill mesh {nx}x{nz}, degree {P} ({m.n_cells * (P + 1) ** 2} pressure "
                  f"DoFs), dt={dt} s, seeded smooth rhs, FGMRES(30) to |b - S p| <= 1e-10 |b|",
        "results": res,
        "speedup_cheb_fp32_vs_fp64_jacobi": res["jacobi"]["solve_s"] / res["cheb_fp32"]["solve_s"],
        "speedup_mg_fp32_vs_mg_fp64": res["mg_fp64"]["solve_s"] / res["mg_fp32"]["solve_s"],
    }
    del op, sol, b
    # ---- IMEX steps: periodic hill 512x256, degree 4, dt 0.5 s; eps 1e-8 (the reference's
    #      default) and eps 1e-10 (tight enough that mixed and FP64 fields agree to <= 1e-8)
    nx, nz, dt, nsteps = 512, 256, 0.5, 3
    m = M.hill_mesh(nx, nz, periodic_x=True)
    st = M.hill_state(m, P, seed=SEED, modes=4)

    def imex_case(eps, names):
        steps, states = {}, {}
        for name, pc in names:
            g = IMEXStepper(m, P, sc.Ma, sc.Fr, dt, eps=eps, schur_preconditioner=pc)
            g.set_state(d(st.rho), d(st.u), d(st.p))
            g.step(1)  # warm-up step
            torch.cuda.synchronize(dev)
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record()
            g.step(nsteps)
            e1.record()
            e1.synchronize()
            steps[name] = {"s_per_step": e0.elapsed_time(e1) * 1e-3 / nsteps, "stats_last_step": g.stats()}
            states[name] = [t.clone() for t in g.get_state()]
            del g
        for name in steps:
            if name != "fp64":  # max over the density, velocity and pressure fields
                steps[name]["rel_error_vs_fp64"] = max(float(torch.linalg.norm(a - b) / torch.linalg.norm(b))
                                                       for a, b in zip(states[name], states["fp64"]))
        return steps, states

    # ---- stage-1 tangent-linear and adjoint (af_imex_stage1_*), same mesh, wall clock
    g = IMEXStepper(m, P, sc.Ma, sc.Fr, dt, eps=1e-10, schur_preconditioner="cheb_fp32")
    x0 = (d(st.rho), d(st.u), d(st.p))
    rng = np.random.default_rng(SEED + 5)
    rnd = lambda v: torch.from_numpy(rng.standard_normal(v.numel()) * float(v.abs().max())).to(dev)
    dx, yb = tuple(rnd(v) for v in x0), tuple(rnd(v) for v in x0)
    g.stage1_forward(*x0)  # warm-up
    torch.cuda.synchronize(dev)
    t0 = time.perf_counter()
    g.stage1_forward(*x0)
    torch.cuda.synchronize(dev)
    t_f = time.perf_counter() - t0
    t0 = time.perf_counter()
    dy = g.stage1_tangent(*dx, rel_tol=1e-10)
    torch.cuda.synchronize(dev)
    t_t = time.perf_counter() - t0
    t0 = time.perf_counter()
    xb = g.stage1_backward(*yb, rel_tol=1e-10)
    torch.cuda.synchronize(dev)
    t_b = time.perf_counter() - t0
    lhs = sum(float(torch.dot(a_, b_)) for a_, b_ in zip(dy, yb))
    rhs = sum(float(torch.dot(a_, b_)) for a_, b_ in zip(dx, xb))
    scl = sum(float((a_.abs() * b_.abs()).sum()) for a_, b_ in zip(dy, yb))
    out["stage1_adjoint"] = {
        "config": f"IMEX stage 1 (density update + pressure fixed point) on the periodic hill {nx}x{nz}, degree {P}, "
                  f"dt={dt} s, forward eps 1e-10, tangent/adjoint Schur solves to 1e-10, seeded random directions",
        "forward_s": t_f, "tangent_s": t_t, "backward_s": t_b,
        "fixed_point_iterations": g.stats()["fixed_point_iterations"][0],
        "dot_product_rel_error": abs(lhs - rhs) / scl,
    }
    del g, dy, xb
    # ---- gradient over many steps with checkpointing (the hill at 256x128, degree 4, 50 steps,
    #      a checkpoint every 10): J = |w|^2 / 2 over the lower 8 km of the final state
    ga, gnx, gnz, gsteps, gevery = None, 256, 128, 50, 10
    gm = M.hill_mesh(gnx, gnz, periodic_x=True)
    gst = M.hill_state(gm, P, seed=SEED, modes=4)
    ga = IMEXStepper(gm, P, sc.Ma, sc.Fr, dt, eps=1e-10, schur_preconditioner="cheb_fp32")
    gx = (d(gst.rho), d(gst.u), d(gst.p))
    zc = M.dof_coordinates(gm, P)[..., 1].reshape(-1)
    low = d((zc < 8000.0).astype(np.float64))
    ga.set_state(*gx)
    torch.cuda.synchronize(dev)
    t0 = time.perf_counter()
    ga.step(gsteps)
    torch.cuda.synchronize(dev)
    t_fwd = time.perf_counter() - t0
    _, uN, _ = ga.get_state()
    nsg = gm.n_cells * (P + 1) ** 2
    wbar = torch.zeros(2 * nsg, dtype=torch.float64, device=dev)
    cells = uN.view(gm.n_cells, 2, (P + 1) ** 2)  # velocity: per cell x then z components
    wbar.view(gm.n_cells, 2, (P + 1) ** 2)[:, 1, :] = cells[:, 1, :] * low.view(gm.n_cells, (P + 1) ** 2)
    zr = torch.zeros(nsg, dtype=torch.float64, device=dev)
    torch.cuda.synchronize(dev)
    t0 = time.perf_counter()
    gb = ga.gradient(*gx, gsteps, gevery, zr, wbar, zr, rel_tol=1e-10)
    torch.cuda.synchronize(dev)
    t_grad = time.perf_counter() - t0
    out["gradient"] = {
        "config": f"hill {gnx}x{gnz} (periodic lateral), degree {P}, dt={dt} s, {gsteps} IMEX steps (mixed precision, "
                  f"eps 1e-10), J = |w|^2/2 over z < 8 km at the final step, gradient with respect to the initial "
                  f"state, a checkpoint every {gevery} steps; wall clock",
        "forward_s": t_fwd, "gradient_s": t_grad, "gradient_over_forward": t_grad / t_fwd,
        "grad_norms": [float(torch.linalg.norm(v)) for v in gb],
    }
    del ga, gb
    # ---- production size: periodic hill 2048x512, p = 4, 104.9 M DoFs,
    #      dt 0.125 s, eps 1e-8, one warm-up and two timed steps per precision
    pm = M.hill_mesh(2048, 512, periodic_x=True)
    pst = M.hill_state(pm, P, seed=SEED, modes=4)
    prod, pstates = {}, {}
    for name, pc in (("fp64", "jacobi"), ("mixed", "cheb_fp32")):
        free0 = torch.cuda.mem_get_info(dev)[0]
        g = IMEXStepper(pm, P, sc.Ma, sc.Fr, 0.125, eps=1e-8, schur_preconditioner=pc)
        g.set_state(d(pst.rho), d(pst.u), d(pst.p))
        g.step(1)
        torch.cuda.synchronize(dev)
        used = free0 - torch.cuda.mem_get_info(dev)[0]
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        g.step(2)
        e1.record()
        e1.synchronize()
        prod[name] = {"s_per_step": e0.elapsed_time(e1) * 1e-3 / 2, "stats_last_step": g.stats(),
                      "device_bytes": int(used)}
        pstates[name] = [t.clone() for t in g.get_state()]
        del g
    prod["mixed"]["rel_error_vs_fp64"] = max(float(torch.linalg.norm(a_ - b_) / torch.linalg.norm(b_))
                                             for a_, b_ in zip(pstates["mixed"], pstates["fp64"]))
    out["production"] = {
        "config": "periodic hill 2048x512, degree 4 (104.9 M DoFs), dt=0.125 s, eps=1e-8, 1 warm-up + 2 timed "
                  "steps; device_bytes: device memory taken by the stepper (state, stage vectors, solver)",
        "results": prod,
        "speedup_mixed_vs_fp64": prod["fp64"]["s_per_step"] / prod["mixed"]["s_per_step"],
    }
    del pstates
    steps, _ = imex_case(1e-8, (("fp64", "jacobi"), ("fp64_cheb", "cheb_fp64"), ("mixed", "cheb_fp32"),
                                ("reference_criterion", -1)))
    tight, tight_states = imex_case(1e-10, (("fp64", "jacobi"), ("fp64_cheb", "cheb_fp64"), ("mixed", "cheb_fp32")))
    out["imex"] = {
        "config": f"periodic hill {nx}x{nz}, degree {P}, dt={dt} s, 1 warm-up + {nsteps} timed steps; "
                  "fp64: Schur FGMRES + Jacobi (FP64); fp64_cheb: Schur FGMRES + the same Chebyshev polynomial "
                  "preconditioner in FP64 (like for like: precision is the only difference to mixed); mixed: "
                  "Schur FGMRES (FP64) + FP32 Chebyshev polynomial preconditioner (degree 20, cell inverses by "
                  "change of basis), all to |b - S p| <= eps |b|; "
                  "reference_criterion: the reference's left-Jacobi GMRES stopping on |D^-1 r| <= eps |b| (a "
                  "looser criterion, shown for scale)",
        "eps": 1e-8,
        "results": steps,
        "speedup_mixed_vs_fp64": steps["fp64"]["s_per_step"] / steps["mixed"]["s_per_step"],
        "speedup_mixed_vs_fp64_cheb": steps["fp64_cheb"]["s_per_step"] / steps["mixed"]["s_per_step"],
        "tight": {
            "eps": 1e-10,
            "results": tight,
            "speedup_mixed_vs_fp64": tight["fp64"]["s_per_step"] / tight["mixed"]["s_per_step"],
            "speedup_mixed_vs_fp64_cheb": tight["fp64_cheb"]["s_per_step"] / tight["mixed"]["s_per_step"],
            "field_error_mixed_vs_fp64": tight["mixed"]["rel_error_vs_fp64"],
            "field_error_mixed_vs_fp64_cheb": max(
                float(torch.linalg.norm(a_ - b_) / torch.linalg.norm(b_))
                for a_, b_ in zip(tight_states["mixed"], tight_states["fp64_cheb"])),
        },
    }
    return out


def run_ours(args, rank, world, local_rank):
    import torch
    import torch.distributed as dist
    from atmospheric_flows_b200 import mesh as M
    from atmospheric_flows_b200.operator import EULEROperator, lib
    import ctypes

    torch.cuda.set_device(local_rank)
    dev = torch.device("cuda", local_rank)
    sc = M.Scaling()
    m, src_h = workload()
    P = DEGREE
    ns = m.n_cells * (P + 1) ** 2
    stream = torch.cuda.Stream(device=dev)
    op = EULEROperator(m, P, sc.Ma, sc.Fr, 2.0, stream=stream)
    op.set_HYPERBOLIC_stage(STAGE)
    src = [torch.from_numpy(a).to(dev) for a in src_h]
    bufs = [torch.empty(k * ns, dtype=torch.float64, device=dev) for k in (1, 2, 1)]

    # ---- device-resident throughput (value)
    for _ in range(args.warmup):
        op.vmult_rhs_fused(*bufs, src)
    stream.synchronize()
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    launches0 = op.launch_count()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with Clocks(gpu_pci_id(dev) or local_rank) as clk:
        clk.mark()
        e0.record(stream)
        for _ in range(args.steps):
            op.vmult_rhs_fused(*bufs, src)
        e1.record(stream)
        e1.synchronize()
        clk.mark()
    torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    t_total = reduce_max_over_ranks(e0.elapsed_time(e1) * 1e-3, world, dev)
    launches = op.launch_count() - launches0
    t_step = t_total / args.steps
    dofs = 4 * ns
    value = dofs * world / t_step / 1e9

    # ---- end to end through the host-buffer C-ABI call (pinned host memory)
    src_pin = [torch.from_numpy(a).pin_memory().numpy() for a in src_h]
    out_pin = [torch.empty(k * ns, dtype=torch.float64).pin_memory().numpy() for k in (1, 2, 1)]
    for _ in range(max(1, args.warmup // 2)):
        op.vmult_rhs_fused_host(*out_pin, src_pin)
    K2 = max(3, min(args.steps, 10))
    if world > 1:
        dist.barrier()
    e2, e3 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e2.record(stream)
    for _ in range(K2):
        op.vmult_rhs_fused_host(*out_pin, src_pin)
    e3.record(stream)
    e3.synchronize()
    t_e2e = reduce_max_over_ranks(e2.elapsed_time(e3) * 1e-3 / K2, world, dev)
    h2d = sum(a.nbytes for a in src_pin)
    d2h = sum(a.nbytes for a in out_pin)
    # parity spot check of the e2e outputs against the device outputs
    assert np.array_equal(out_pin[2], bufs[2].cpu().numpy())

    # ---- roofline
    peak, kind = measured_peaks()
    alg_bytes = 8 * ns * 11  # 7 scalar fields in, 4 out
    prof = profile_numbers()
    fp64_peak = ctypes.c_double()
    lib().af_measure_fp64_peak(ctypes.byref(fp64_peak))
    roofline = {"bound": "hbm", "achieved": alg_bytes / t_step / 1e9, "peak": peak, "unit": "GB/s",
                "frac": alg_bytes / t_step / 1e9 / peak, "traffic": prof.get("traffic_bytes_per_launch"),
                "peak_source": f"{kind} (MEASURED_PEAKS.json hbm_gbs)" if kind == "measured" else "fallback",
                "alg_bytes_per_launch": alg_bytes}
    if "fp64_flops_per_launch" in prof:
        ach = prof["fp64_flops_per_launch"] / t_step / 1e12
        roofline["fp64"] = {"achieved_tflops": ach, "peak_tflops": fp64_peak.value, "frac": ach / fp64_peak.value,
                            "flops_per_launch": prof["fp64_flops_per_launch"],
                            "note": "executed FP64 flops per launch from ncu; peak measured by af_measure_fp64_peak"}
        # the same figures as flat keys beside the HBM ones (the kernel is FP64-bound, not HBM-bound)
        roofline["fp64_achieved_tflops"] = ach
        roofline["fp64_peak_tflops"] = fp64_peak.value
        roofline["fp64_frac"] = ach / fp64_peak.value

    line = None
    if rank == 0:
        # ---- degree sweep (same mesh), device-resident
        # the sweep, the solver measurements and the CPU baseline belong to the 1-GPU line; at
        # N > 1 the line carries the replicated apply and its end-to-end time only
        extras = world == 1
        sweep = {}
        if not args.no_sweep and extras:
            for Pd in (2, 3, 4, 5, 6):
                md, sh = workload(Pd, modes=4)
                nsd = md.n_cells * (Pd + 1) ** 2
                opd = EULEROperator(md, Pd, sc.Ma, sc.Fr, 2.0, stream=stream)
                opd.set_HYPERBOLIC_stage(STAGE)
                sd = [torch.from_numpy(a).to(dev) for a in sh]
                bd = [torch.empty(k * nsd, dtype=torch.float64, device=dev) for k in (1, 2, 1)]
                td = time_device(opd, bd, sd, stream, 10, 3)
                sweep[str(Pd)] = {"gdofs": 4 * nsd / td / 1e9, "us_per_apply": td * 1e6,
                                  "hbm_frac": 8 * nsd * 11 / td / 1e9 / peak}
                del opd, sd, bd
        # ---- tangent and backward of the same apply (device-resident, same inputs)
        rng = np.random.default_rng(SEED + 3)
        dsrc = [torch.from_numpy(rng.standard_normal(a.size)).to(dev) for a in src_h]
        ybar = [torch.from_numpy(rng.standard_normal(k * ns)).to(dev) for k in (1, 2, 1)]
        xbar = [torch.empty(a.size, dtype=torch.float64, device=dev) for a in src_h]
        dy = [torch.empty(k * ns, dtype=torch.float64, device=dev) for k in (1, 2, 1)]

        def timed(fn, K=10, W=3):
            for _ in range(W):
                fn()
            stream.synchronize()
            a0, a1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a0.record(stream)
            for _ in range(K):
                fn()
            a1.record(stream)
            a1.synchronize()
            return a0.elapsed_time(a1) * 1e-3 / K
        t_tan = timed(lambda: op.vmult_rhs_fused_tangent(src, dsrc, *dy))
        t_bwd = timed(lambda: op.vmult_rhs_fused_backward(src, *ybar, xbar))
        autodiff = {"forward_ms": t_step * 1e3, "tangent_ms": t_tan * 1e3, "backward_ms": t_bwd * 1e3,
                    "backward_over_forward": t_bwd / t_step,
                    "note": "af_vmult_rhs_fused_tangent / _backward on the bench workload (one launch each)"}
        solvers = {} if (args.no_solvers or not extras) else run_solvers(dev)
        threads = os.cpu_count() or 1
        cpu_v = None
        if extras:
            cm, csrc = cpu_sample()
            cpu_v = 4 * cm.n_cells * (DEGREE + 1) ** 2 / time_cpu_port(cm, csrc, 2, 20, threads) / 1e9
        parity = strip_parity(dev, stream)
        line = {"metric": METRIC, "value": value, "unit": "GDoF/s", "n_gpus": world, "steps": args.steps,
                "warmup": args.warmup, "ms_per_step": t_step * 1e3, "higher_is_better": True, "scaling": "weak",
                "vs_baseline": None, "dtype": "f64",
                "data": "synthetic (hydrostatic background + seeded Fourier perturbation)", "config": config(),
                "e2e": {"value": dofs * world / t_e2e / 1e9, "unit": "GDoF/s", "h2d_bytes_per_step": h2d,
                        "d2h_bytes_per_step": d2h, "ms_per_step": t_e2e * 1e3,
                        "call": "af_vmult_rhs_fused_host (pinned host buffers)"},
                "roofline": roofline, "gpu_launches": launches,
                "clocks": clk.summary(),
                "cpu_baseline": ({"value": cpu_v, "unit": "GDoF/s", "cores": threads, "kind": "port",
                                  "sample": cpu_sample_label(), "note": CPU_NOTE} if extras else None),
                "parity_rel_l2": parity,
                "parity_check": f"GPU fused apply vs the oracle on the {NX}x{CPU_ROWS} CPU-sample strip (same mesh "
                                "and inputs on both sides), largest relative L2 error over the three outputs",
                "degree_sweep": sweep, "autodiff": autodiff, **solvers}
        print(json.dumps(line), flush=True)
    return line


def reduce_max_over_ranks(value, world, device):
    """The maximum of a per-rank time over all ranks (all ranks call it, in the same order)."""
    if world <= 1:
        return value
    import torch
    import torch.distributed as dist
    t = torch.tensor([value], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def run_profile_case(kind):
    """A short run of one workload for ncu captures (no timing, no JSON): 'rhs' the fused
    stage-1 apply, 'adjoint' its tangent and backward, 'schur' the FP32 multigrid setup and
    one V-cycle on the 1024x256 pressure system, 'imex' two mixed-precision IMEX steps on the
    periodic 512x256 hill."""
    import torch
    from atmospheric_flows_b200 import mesh as M
    from atmospheric_flows_b200.operator import EULEROperator
    sc = M.Scaling()
    d = lambda a: torch.from_numpy(np.ascontiguousarray(a)).cuda()
    if kind == "imex":
        from atmospheric_flows_b200.imex import IMEXStepper
        m = M.hill_mesh(512, 256, periodic_x=True)
        st = M.hill_state(m, DEGREE, seed=SEED, modes=4)
        g = IMEXStepper(m, DEGREE, sc.Ma, sc.Fr, 0.5, schur_preconditioner="cheb_fp32")
        g.set_state(d(st.rho), d(st.u), d(st.p))
        g.step(2)
        torch.cuda.synchronize()
        return
    if kind in ("rhs", "adjoint"):
        m, src_h = workload(DEGREE, modes=2)
        op = EULEROperator(m, DEGREE, sc.Ma, sc.Fr, 2.0)
        op.set_stream(torch.cuda.current_stream())
        op.set_HYPERBOLIC_stage(1)
        ns = m.n_cells * (DEGREE + 1) ** 2
        src = [d(a) for a in src_h]
        dy = [torch.empty(k * ns, dtype=torch.float64, device="cuda") for k in (1, 2, 1)]
        for _ in range(2):
            op.vmult_rhs_fused(*dy, src)
        if kind == "adjoint":
            yb = [d(np.random.default_rng(1).standard_normal(k * ns)) for k in (1, 2, 1)]
            xb = [torch.empty_like(a) for a in src]
            op.vmult_rhs_fused_tangent(src, src, *dy)
            op.vmult_rhs_fused_backward(src, *yb, xb)
    else:
        from atmospheric_flows_b200.schur import SchurSolver
        m = M.hill_mesh(1024, 256)
        st = M.hill_state(m, DEGREE, modes=2)
        op = EULEROperator(m, DEGREE, sc.Ma, sc.Fr, 0.5)
        op.set_stream(torch.cuda.current_stream())
        op.set_schur_mode(1)
        op.set_HYPERBOLIC_stage(1)
        op.set_rho_for_fixed(d(st.rho))
        op.set_pres_fixed(d(st.p))
        op.set_NS_stage(2)
        s = SchurSolver(op, "mg_fp32", smoother_degree=5)
        s.setup()
        z = torch.empty(m.n_cells * (DEGREE + 1) ** 2, dtype=torch.float64, device="cuda")
        s.precondition(z, d(st.p))
    torch.cuda.synchronize()


def run_timeline():
    """One warm IMEX step (periodic 512x256 hill, degree 4, dt 0.5 s, eps 1e-8) with the mixed
    and the FP64 solver, recorded by the CUDA activity tracer of torch.profiler: the device
    time of every kernel and copy in the step, the span from the first start to the last end,
    the busy time (union of the intervals), the idle gaps between them, and the kernels with
    the most device time.  Warm-cache and in-stream, unlike an ncu launch list.  Prints one
    JSON object; the tracer's own overhead makes the step a little longer than in the
    timed bench."""
    import torch
    from torch.profiler import ProfilerActivity, profile
    from atmospheric_flows_b200 import mesh as M
    from atmospheric_flows_b200.imex import IMEXStepper
    sc = M.Scaling()
    m = M.hill_mesh(512, 256, periodic_x=True)
    st = M.hill_state(m, DEGREE, seed=SEED, modes=4)
    d = lambda a: torch.from_numpy(np.ascontiguousarray(a)).cuda()
    out = {"config": "periodic hill 512x256, degree 4, dt=0.5 s, eps=1e-8, one warm step after one warm-up step; "
                     "step_backward: the adjoint of one mixed-precision step (eps 1e-10, as in the gradient) at its "
                     "recorded forward, after one warm-up adjoint"}

    def trace(fn):
        torch.cuda.synchronize()
        with profile(activities=[ProfilerActivity.CUDA]) as prof:
            fn()
            torch.cuda.synchronize()
        iv = sorted((e.time_range.start, e.time_range.end, e.name) for e in prof.events()
                    if e.device_type == torch.autograd.DeviceType.CUDA)
        busy, cs, ce = 0.0, None, None
        for s0, e0, _ in iv:
            if ce is None or s0 > ce:
                busy += 0.0 if ce is None else ce - cs
                cs, ce = s0, e0
            else:
                ce = max(ce, e0)
        busy += 0.0 if ce is None else ce - cs
        gaps = np.array([iv[i + 1][0] - iv[i][1] for i in range(len(iv) - 1)])
        agg = {}
        for s0, e0, name in iv:
            a = agg.setdefault(name, [0, 0.0])
            a[0] += 1
            a[1] += e0 - s0
        span = iv[-1][1] - iv[0][0]
        top = sorted(agg.items(), key=lambda kv: -kv[1][1])[:16]
        return {
            "device_events": len(iv), "span_ms": span / 1e3, "busy_ms": busy / 1e3,
            "idle_ms": float(gaps[gaps > 0].sum()) / 1e3, "gap_median_us": float(np.median(gaps)),
            "gaps_over_20us": int((gaps > 20).sum()),
            "top": [{"kernel": k[:160], "launches": v[0], "total_ms": round(v[1] / 1e3, 3),
                     "per_launch_us": round(v[1] / v[0], 1), "share": round(v[1] / busy, 4)} for k, v in top],
        }

    for label, pc in (("mixed", "cheb_fp32"), ("fp64", "jacobi")):
        g = IMEXStepper(m, DEGREE, sc.Ma, sc.Fr, 0.5, eps=1e-8, schur_preconditioner=pc)
        g.set_state(d(st.rho), d(st.u), d(st.p))
        g.step(1)
        out[label] = trace(lambda: g.step(1))
        del g
        torch.cuda.synchronize()
    g = IMEXStepper(m, DEGREE, sc.Ma, sc.Fr, 0.5, eps=1e-10, schur_preconditioner="cheb_fp32")
    x = (d(st.rho), d(st.u), d(st.p))
    g.step_forward(*x)
    yb = tuple(torch.ones_like(v) for v in x)
    g.step_backward(*yb, rel_tol=1e-10)
    out["step_backward"] = trace(lambda: g.step_backward(*yb, rel_tol=1e-10))
    del g
    torch.cuda.synchronize()
    print(json.dumps(out))


def run_production_full(nsteps=1000, adjoint_steps=100, every=10):
    """The production-size hill run in full (opt-in: about half an hour on one B200): periodic
    hill 2048x512, degree 4 (104.9 M DoFs), dt 0.125 s, eps 1e-8; nsteps mixed-precision steps
    and nsteps plain FP64 steps from the same state, the field error between them, and the
    adjoint gradient of J = |w|^2/2 over z < 8 km at the final step with respect to the state
    adjoint_steps steps earlier, by checkpointed recomputation (a checkpoint every `every`
    steps).  Device time by CUDA events for the steps; wall clock for the gradient."""
    import torch
    from atmospheric_flows_b200 import mesh as M
    from atmospheric_flows_b200.imex import IMEXStepper
    sc = M.Scaling()
    P = DEGREE
    d = lambda a: torch.from_numpy(np.ascontiguousarray(a)).cuda()
    m = M.hill_mesh(2048, 512, periodic_x=True)
    st = M.hill_state(m, P, seed=SEED, modes=4)
    out = {"config": f"periodic hill 2048x512, degree {P} ({4 * m.n_cells * (P + 1) ** 2} DoFs), dt=0.125 s, eps=1e-8, "
                     f"{nsteps} steps per precision from the same state; gradient of J = |w|^2/2 over z < 8 km at step "
                     f"{nsteps} with respect to the state at step {nsteps - adjoint_steps}, a checkpoint every {every}"}
    finals = {}
    for name, pc in (("mixed", "cheb_fp32"), ("fp64", "jacobi")):
        g = IMEXStepper(m, P, sc.Ma, sc.Fr, 0.125, eps=1e-8, schur_preconditioner=pc)
        g.set_state(d(st.rho), d(st.u), d(st.p))
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        start_state = None
        e0.record()
        g.step(nsteps - adjoint_steps)
        if name == "mixed":
            start_state = [t.clone() for t in g.get_state()]
        g.step(adjoint_steps)
        e1.record()
        e1.synchronize()
        finals[name] = [t.clone() for t in g.get_state()]
        out[name] = {"s_per_step": e0.elapsed_time(e1) * 1e-3 / nsteps, "stats_last_step": g.stats()}
        if name == "mixed":
            zc = M.dof_coordinates(m, P)[..., 1].reshape(-1)
            low = d((zc < 8000.0).astype(np.float64))
            uN = finals[name][1]
            ns = m.n_cells * (P + 1) ** 2
            wbar = torch.zeros(2 * ns, dtype=torch.float64, device="cuda")
            wbar.view(m.n_cells, 2, -1)[:, 1, :] = uN.view(m.n_cells, 2, -1)[:, 1, :] * low.view(m.n_cells, -1)
            zr = torch.zeros(ns, dtype=torch.float64, device="cuda")
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            gb = g.gradient(*start_state, adjoint_steps, every, zr, wbar, zr, rel_tol=1e-10)
            torch.cuda.synchronize()
            out["gradient"] = {"seconds": time.perf_counter() - t0, "steps": adjoint_steps, "checkpoint_every": every,
                               "grad_norms": [float(torch.linalg.norm(v)) for v in gb],
                               "finite": all(bool(torch.isfinite(v).all()) for v in gb)}
            del gb, start_state
        del g
        torch.cuda.synchronize()
    out["field_error_mixed_vs_fp64"] = max(float(torch.linalg.norm(a - b) / torch.linalg.norm(b))
                                           for a, b in zip(finals["mixed"], finals["fp64"]))
    out["speedup_mixed_vs_fp64"] = out["fp64"]["s_per_step"] / out["mixed"]["s_per_step"]
    print(json.dumps(out), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=2000)  # about 0.9 s of timed applies at 512x256, p = 4
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--no-sweep", action="store_true")
    ap.add_argument("--no-solvers", action="store_true", help="skip the Schur-solve and IMEX-step measurements")
    ap.add_argument("--profile", choices=["rhs", "adjoint", "schur", "imex"],
                    help="run one workload briefly for an ncu capture and exit (no measurement)")
    ap.add_argument("--production-full", action="store_true",
                    help="the 2048x512 hill run in full: 1000 mixed and 1000 FP64 steps, the gradient over the last "
                         "100 (about half an hour); prints one JSON object")
    ap.add_argument("--timeline", action="store_true",
                    help="trace one warm IMEX step (mixed and FP64) and print its kernel timeline summary")
    args = ap.parse_args()
    if args.profile:
        run_profile_case(args.profile)
        return
    if args.timeline:
        run_timeline()
        return
    if args.production_full:
        run_production_full()
        return
    args.warmup = max(3, args.warmup)
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        run_reference(args, rank)
        return
    if world > 1:
        import datetime
        import torch
        import torch.distributed as dist
        torch.cuda.set_device(local_rank)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    try:
        run_ours(args, rank, world, local_rank)
    finally:
        if world > 1:
            import torch.distributed as dist
            dist.destroy_process_group()


if __name__ == "__main__":
    main()
