"""Benchmark: grid-point RK4 updates/s of the BSSN + dust evolution on B200.

Workload (default): one periodic BSSN + pressureless-dust box of 256^3 points
per GPU, 8th-order stencils, harmonic lapse, FP64 (reference operand order).
A "step" is one full RK4 step (4 fused substep launches) of that box; each
rank evolves its own box (independent replicas, weak scaling).  Inputs are
synthetic: the seeded Gaussian-random-field dust initial data (rms density
contrast 1e-4, P(k) ~ k^0.96 with a Gaussian cutoff at N/4, synchronous gauge,
constraint-satisfying), generated on the host.  The other precisions of the
same kernel (fp64_fma, mixed) are timed on the same box and state their field
and Hamiltonian-constraint error against the FP64 run after the same steps.

Printed JSON (rank 0, one line): value = whole-job updates/s with the state
resident in HBM; e2e = the same through the C ABI with the full state copied
host->device and device->host around every step (pinned buffers; the next
step's input comes in and the previous step's result goes out while a step
runs: cg_prefetch_state_async + cg_exchange_state_async);
roofline = the substep
kernel's algorithmic HBM bytes against the measured copy bandwidth;
cpu_baseline = the reference's own sources (oracle/_ref) on the host cores.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import threading
import time
from pathlib import Path

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

# Algorithmic HBM bytes per grid-point RK4 update of the fused FP64 scheme,
# each value counted once (perfect stencil reuse): substep 1 reads p, writes f
# and a^2 (3E); substeps 2-3 read a, p, f and write f, a (5E each); substep 4
# reads a, p, f and writes p (4E): 17E values, E = 22 evolved fields, plus the
# reference's lagged dust quantities W, sqrt(gamma), g_ij (8 values written at
# substeps 1-3 and read at 2-4, 48 values): 422 values = 3376 bytes.
ALGO_BYTES_PER_UPDATE = {"dust": 3376, "scalar": 3128, "vacuum": 17 * 18 * 8}
# FP32-mixed layout, same counting rule: per field the stage inputs a are FP32
# (substep 1: p 8 + f 8 + a 4; substeps 2-3: a 4 + p 8 + f 8 + f 8 + a 4;
# substep 4: a 4 + p 8 + f 8 + p 8 = 112 B) and the lagged dust quantities
# are recomputed from the previous substep's FP32 input (11 values read at
# substeps 2-4): 22 * 112 + 3 * 11 * 4 = 2596 bytes.
ALGO_BYTES_MIXED_DUST = 22 * 112 + 3 * 11 * 4


def algo_bytes(precision: str) -> int:
    return ALGO_BYTES_MIXED_DUST if precision == "mixed" else ALGO_BYTES_PER_UPDATE["dust"]


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--n", type=int, default=256)
    ap.add_argument("--order", type=int, default=8)
    ap.add_argument("--precision", default="fp64", choices=["fp64", "fp64_fma", "mixed"])
    ap.add_argument("--e2e-steps", type=int, default=10)
    ap.add_argument("--cpu-baseline", type=int, default=1, help="time the reference CPU build (rank 0)")
    ap.add_argument("--ncu", action="store_true", help="short run for profiler capture (no JSON extras)")
    ap.add_argument("--variants", default="fp64_fma,mixed", help="comma list of extra precisions timed alongside")
    ap.add_argument("--ensemble", type=int, default=1, help="also time the 48-box ensemble (variants.ensemble)")
    ap.add_argument("--scalar", type=int, default=1, help="also time the GRF scalar configuration (variants.scalar)")
    ap.add_argument("--workload", choices=["box", "ensemble", "slab"], default="box",
                    help="box: one 256^3 box per GPU; ensemble: 48 boxes of 32^3/64^3/96^3 split over the GPUs; "
                         "slab: one (256 N) x 256 x 256 box cut into N x-slabs with a ghost exchange per substep")
    return ap.parse_args()


def dist_setup(a):
    import torch

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import torch.distributed as dist
        from datetime import timedelta

        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=timedelta(seconds=600), device_id=torch.device("cuda", local))
    else:
        torch.cuda.set_device(0)
    return world, rank, local


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu: int):
        self.gpu = gpu
        self.rows = []
        self._stop = threading.Event()
        self._t = threading.Thread(target=self._run, daemon=True)

    def _run(self):
        while not self._stop.is_set():
            try:
                out = subprocess.run(["nvidia-smi", "-i", str(self.gpu), f"--query-gpu={self.Q}",
                                      "--format=csv,noheader,nounits"], capture_output=True,
                                     text=True, timeout=5).stdout.strip()
                if out:
                    self.rows.append([x.strip() for x in out.split(",")])
            except Exception:
                pass
            self._stop.wait(0.2)

    def __enter__(self):
        self._t.start()
        return self

    def __exit__(self, *exc):
        self._stop.set()
        self._t.join(timeout=10)

    def summary(self):
        if not self.rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unavailable"]}
        sm = [float(r[1]) for r in self.rows if r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in self.rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in self.rows for i in range(4) if len(r) > 5 + i and r[5 + i] == "Active"})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(self.rows)}


def measured_peaks():
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        d = json.loads(p.read_text())
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def profiled_traffic(n: int, order: int, precision: str):
    """DRAM bytes per substep launch from the committed ncu summary, or None."""
    prof = ROOT / "profiles" / "stage_kernel_traffic.json"
    try:
        return json.loads(prof.read_text()).get(f"{n}_{order}_{precision}")
    except Exception:
        return None


def profiled_flops(precision: str):
    """FP64 flops per grid-point RK4 update of the substep kernel (four
    launches), counted by ncu (dadd + dmul + 2 dfma, thread level) and
    committed in profiles/stage_kernel_traffic.json; None if absent."""
    prof = ROOT / "profiles" / "stage_kernel_traffic.json"
    try:
        return json.loads(prof.read_text()).get("fp64_flops_per_update", {}).get(precision)
    except Exception:
        return None


def fp64_peak(L) -> float | None:
    """This GPU's FP64 flop/s, measured by the library (cg_fp64_peak)."""
    import ctypes

    v = ctypes.c_double()
    return v.value if L.cg_fp64_peak(ctypes.byref(v)) == 0 else None


def make_state(n: int, seed: int, order: int, gpu: bool = True):
    """GRF dust initial data: the random field drawn on the host, the
    construction on the GPU (the host construction when gpu=False); both give
    the same data to rounding."""
    from cosmograph_b200 import ics

    if gpu:
        return ics.grf_dust_gpu(n, seed=seed, rms_delta=1.0e-4, order=order, host_delta=True)
    return ics.grf_dust(n, seed=seed, rms_delta=1.0e-4, order=order)


def accuracy(ref, got, h_ref, h_got) -> dict:
    """Per-field max|got - ref| / max|ref - mean(ref)| (fields with a nonzero
    spread) and the Hamiltonian-constraint L2 norms of both runs."""
    import numpy as np

    worst, wname = 0.0, None
    for f, name in enumerate(ref.names):
        r = ref.fields[f]
        spread = float(np.abs(r - r.mean()).max())
        if spread == 0.0:
            continue
        e = float(np.abs(got.fields[f] - r).max()) / spread
        if e > worst:
            worst, wname = e, name
    return {"field_err_rel_perturbation": worst, "worst_field": wname,
            "H_L2": float(h_got["H"][7]), "H_L2_fp64": float(h_ref["H"][7]),
            "H_ratio": float(h_got["H"][7] / h_ref["H"][7]),
            "M_L2": float(h_got["M"][7]), "M_L2_fp64": float(h_ref["M"][7])}


def box_config(n: int, order: int, precision: str, world: int) -> dict:
    """The workload description both arms print (ours and --impl reference)."""
    state_gb = 22 * n ** 3 * 8 / 1e9
    return {"workload": f"bssn_dust_{n}cubed_o{order}", "n": n, "stencil_order": order, "lapse": "Harmonic",
            "precision": precision, "boxes_per_gpu": 1, "parallelism": f"replicas x{world}",
            "l2": "inputs larger than L2 (state %.1f GB per box)" % state_gb}


def ensemble_config(specs, world: int, groups=None) -> dict:
    all_pts = sum(s.points for s in specs)
    state_gb = 22 * all_pts * 8 / 1e9
    d = {"workload": "ensemble_48_boxes_16x32c_16x64c_16x96c_o4_mixed", "boxes": len(specs),
         "points": all_pts, "stencil_order": 4, "lapse": "Harmonic", "precision": "mixed",
         "seeds": f"{specs[0].seed}..{specs[-1].seed}", "parallelism": f"boxes split over {world} ranks",
         "l2": "inputs larger than L2 (ensemble state %.1f GB)" % state_gb}
    return d


def _reference_steps(binp: Path, st, steps: int, threads: int, timeout: float = 1800.0):
    """Runs an oracle/_ref binary for `steps` RK4 steps of `st`; returns the
    per-step seconds of its step loop (timed like _timer["RK_steps"])."""
    with tempfile.TemporaryDirectory(prefix="cg_bench_cpu_") as tmp:
        tmp = Path(tmp)
        (tmp / "config.txt").write_text("lapse = Harmonic\n")
        st.save(tmp / "in.bin")
        env = dict(os.environ, OMP_NUM_THREADS=str(threads))
        proc = subprocess.run([str(binp), "evolve", str(tmp / "config.txt"), str(tmp / "in.bin"),
                               str(tmp / "out.bin"), str(steps)], capture_output=True, text=True, env=env,
                              timeout=timeout)
    if proc.returncode != 0:
        raise RuntimeError(f"{binp.name} failed ({proc.returncode}): {proc.stderr[-300:]}")
    return [float(l.split()[2]) for l in proc.stdout.splitlines() if l.startswith("CGSTEP")]


def cpu_baseline(st, order: int, steps: int = 3):
    """The reference's own sources on the host cores (oracle/_ref, fast build):
    `steps` RK4 steps of the same box on all host threads, plus the 1-thread
    rate of the same physics on a 64^3 box of the same order (a full 256^3
    step on one thread takes minutes)."""
    from oracle import build_ref

    nx, ny, nz = st.shape
    binp = build_ref.binary_path(nx, ny, nz, order, "fast")
    threads = os.cpu_count() or 1
    if not binp.exists():
        return None
    t0 = time.time()
    step_s = _reference_steps(binp, st, steps, threads)
    wall = time.time() - t0
    if not step_s:
        return None
    rate = nx * ny * nz * len(step_s) / sum(step_s)
    out = {"value": rate, "unit": "grid-pt RK4 updates/s", "cores": threads, "kind": "reference",
           "sample": f"{len(step_s)} RK4 steps of the same {nx}x{ny}x{nz} order-{order} BSSN+dust box, reference "
                     f"sources built -O3 -ffast-math -march=x86-64-v3 -fopenmp ({binp.name}); "
                     f"{sum(step_s):.2f} s of step loop, {wall:.1f} s wall; per step "
                     + ", ".join(f"{s:.2f}" for s in step_s) + " s"}
    one = build_ref.binary_path(64, 64, 64, order, "fast")
    if one.exists():
        small = make_state(64, seed=1, order=order, gpu=False)
        s1 = _reference_steps(one, small, 2, 1)
        if s1:
            out["one_thread"] = {"value": 64 ** 3 * len(s1) / sum(s1), "unit": "grid-pt RK4 updates/s",
                                 "cores": 1, "sample": f"{len(s1)} RK4 steps of a 64^3 order-{order} BSSN+dust "
                                                       f"GRF box on one thread ({one.name})"}
    return out


def ensemble_variant(a, world, rank, stream):
    """The 48-box ensemble (16 each of 32^3, 64^3, 96^3
    BSSN + dust boxes, order 4, FP32-mixed, one autotuned launch per
    substep) timed beside the default box: updates/s over all ranks, the
    launch groups the autotuner chose, and every box against an FP64 run of
    the same steps (worst field error against its spread, Hamiltonian L2
    ratio)."""
    import torch
    import torch.distributed as dist

    from cosmograph_b200 import ensemble
    from cosmograph_b200.evolution import BoxConfig, Evolution

    specs = ensemble.standard_ensemble()
    mine = ensemble.local_share(specs, rank, world)
    states = ensemble.initial_states(mine, order=4, gpu=True)
    all_pts = sum(s.points for s in specs)
    cfg = BoxConfig(order=4, lapse="Harmonic", precision="mixed")
    ev = Evolution(states, [cfg] * len(states))
    ev.set_stream(stream.cuda_stream)
    ev.step(max(a.warmup, 0))
    ev.synchronize()
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    ev.step(a.steps)
    e1.record(stream)
    torch.cuda.synchronize()
    ev.synchronize()
    ms = e0.elapsed_time(e1)
    if world > 1:
        t = torch.tensor([ms], dtype=torch.float64, device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms = float(t.item())
    # the same boxes looped with one launch per box and substep (no batching)
    single = Evolution(states, [cfg] * len(states))
    single.set_option("batch", 0)
    single.set_stream(stream.cuda_stream)
    single.step(max(a.warmup, 0))
    single.synchronize()
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    s0, s1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    s0.record(stream)
    single.step(a.steps)
    s1.record(stream)
    torch.cuda.synchronize()
    single.synchronize()
    ms_single = s0.elapsed_time(s1)
    if world > 1:
        t = torch.tensor([ms_single], dtype=torch.float64, device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms_single = float(t.item())
    single.close()
    fp64 = Evolution(states, [BoxConfig(order=4, lapse="Harmonic")] * len(states))
    fp64.set_stream(stream.cuda_stream)
    fp64.step(max(a.warmup, 0) + a.steps)
    fp64.synchronize()
    acc = {}
    for q, sp in enumerate(mine):
        acc[sp.box_id] = accuracy(fp64.download(q), ev.download(q), fp64.constraints(q), ev.constraints(q))
    groups = ev.groups()
    fp64.close()
    ev.close()
    acc_all = ensemble.gather(acc, world)
    return {"workload": ensemble_config(specs, world)["workload"], "value": all_pts * a.steps / (ms / 1e3),
            "ms_per_step": ms / a.steps, "groups": groups,
            "single_launches": {"value": all_pts * a.steps / (ms_single / 1e3), "ms_per_step": ms_single / a.steps},
            "speedup_vs_single_launches": ms_single / ms,
            "accuracy_vs_fp64": {
                "max_field_err_rel_perturbation": max(v["field_err_rel_perturbation"] for v in acc_all.values()),
                "max_H_ratio": max(v["H_ratio"] for v in acc_all.values()),
                "min_H_ratio": min(v["H_ratio"] for v in acc_all.values()), "boxes": len(acc_all)}}


def scalar_variant(a, world, rank, stream):
    """The GRF scalar configuration timed beside the default box: BSSN + a
    minimally coupled scalar field with V = m^2 phi^2 / 2 (m = 1), phi0 = 1e-2
    plus a k^-3 fluctuation of rms 1e-5 cut off at N/4 (initial data built on
    the GPU, cg_ic_grf_scalar), the box's N and order, harmonic lapse; FP64
    and FP32-mixed updates/s over all ranks, and the mixed run against the
    FP64 run of the same steps (scalar-field error over the fluctuation rms,
    worst field error against its spread, Hamiltonian L2 ratio)."""
    import numpy as np
    import torch
    import torch.distributed as dist

    from cosmograph_b200 import ics
    from cosmograph_b200.evolution import BoxConfig, Evolution

    st = ics.grf_scalar_gpu(a.n, seed=21 + rank, phi0=1e-2, rms=1e-5, mass=1.0, order=a.order)
    out, final = {}, {}
    for prec in ("fp64", "mixed"):
        cfg = BoxConfig(order=a.order, lapse="Harmonic", precision=prec, potential="quadratic", pot_mass=1.0)
        with Evolution(st, cfg) as ev:
            ev.set_stream(stream.cuda_stream)
            ev.step(max(a.warmup, 0))
            ev.synchronize()
            if world > 1:
                dist.barrier()
            torch.cuda.synchronize()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            ev.step(a.steps)
            e1.record(stream)
            torch.cuda.synchronize()
            ev.synchronize()
            ms = e0.elapsed_time(e1)
            if world > 1:
                t = torch.tensor([ms], dtype=torch.float64, device="cuda")
                dist.all_reduce(t, op=dist.ReduceOp.MAX)
                ms = float(t.item())
            out[prec] = {"value": world * a.n ** 3 * a.steps / (ms / 1e3), "ms_per_step": ms / a.steps}
            final[prec] = (ev.download(0), ev.constraints(0))
    acc = accuracy(final["fp64"][0], final["mixed"][0], final["fp64"][1], final["mixed"][1])
    f = st.names.index("phi")
    acc["phi_err_rel_fluctuation"] = float(np.abs(final["mixed"][0].fields[f] - final["fp64"][0].fields[f]).max()) / 1e-5
    out["mixed"]["speedup_vs_fp64"] = out["fp64"]["ms_per_step"] / out["mixed"]["ms_per_step"]
    out["mixed"]["accuracy_vs_fp64"] = acc
    out["workload"] = (f"BSSN + scalar field, {a.n}^3, order {a.order}, V = m^2 phi^2/2 (m = 1), phi0 = 1e-2, "
                       f"k^-3 fluctuation rms 1e-5, {world} box(es)")
    return out


def run_ensemble(a, world, rank, local):
    """--workload ensemble: 48 independent BSSN + dust boxes (16 each of 32^3,
    64^3, 96^3), order 4, FP32-mixed, seeded GRF initial data with rms delta
    log-uniform in [1e-5, 1e-3]; the boxes are split across ranks (no data-path
    communication).  value: updates/s of the batched launch (one launch per
    substep, autotuned); variants: the boxes' own launches, CUDA-graph replay;
    accuracy: every box against an FP64 run of the same steps."""
    import ctypes

    import numpy as np
    import torch
    import torch.distributed as dist

    from cosmograph_b200 import ensemble
    from cosmograph_b200.evolution import BoxConfig, Evolution

    specs = ensemble.standard_ensemble()
    mine = ensemble.local_share(specs, rank, world)
    states = ensemble.initial_states(mine, order=4, gpu=True)
    pts = sum(s.fields[0].size for s in states)
    all_pts = sum(s.points for s in specs)
    cfg = BoxConfig(order=4, lapse="Harmonic", precision="mixed")
    stream = torch.cuda.Stream()

    def barrier():
        if world > 1:
            dist.barrier()

    def max_over_ranks(x):
        if world == 1:
            return x
        t = torch.tensor([x], dtype=torch.float64, device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        return float(t.item())

    def timed(opts, steps, clk=None):
        ev = Evolution(states, [cfg] * len(states))
        for k, v in opts.items():
            ev.set_option(k, v)
        ev.set_stream(stream.cuda_stream)
        ev.step(max(a.warmup, 0))
        ev.synchronize()
        barrier()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        if clk:
            clk.__enter__()
        e0.record(stream)
        ev.step(steps)
        e1.record(stream)
        torch.cuda.synchronize()
        if clk:
            clk.__exit__(None, None, None)
        ev.synchronize()
        barrier()
        return ev, max_over_ranks(e0.elapsed_time(e1))

    clk = ClockSampler(local)
    ev, ms = timed({}, a.steps, clk)
    groups = ev.groups()
    value = all_pts * a.steps / (ms / 1e3)
    # accuracy: each box against an FP64 run of the same warm-up + timed steps
    fp64 = Evolution(states, [BoxConfig(order=4, lapse="Harmonic")] * len(states))
    fp64.set_stream(stream.cuda_stream)
    fp64.step(max(a.warmup, 0) + a.steps)
    fp64.synchronize()
    acc = {}
    for q, s in enumerate(mine):
        ref, got = fp64.download(q), ev.download(q)
        hr, hg = fp64.constraints(q), ev.constraints(q)
        acc[s.box_id] = {**accuracy(ref, got, hr, hg), "n": s.n, "rms_delta": s.rms_delta}
    fp64.close()
    # end to end: every box's state host -> device, one step, device -> host
    h_in = [torch.from_numpy(st.fields.reshape(-1)).pin_memory() for st in states]
    h_out = [torch.empty_like(h).pin_memory() for h in h_in]
    dp = ctypes.POINTER(ctypes.c_double)
    L = ev.L

    def p(h):
        return ctypes.cast(h.data_ptr(), dp)

    def exchange_all():
        for b, (hi, ho) in enumerate(zip(h_in, h_out)):
            ev._check(L.cg_prefetch_state_async(ev.ctx, b, p(hi), hi.numel()))
        for b, (hi, ho) in enumerate(zip(h_in, h_out)):
            ev._check(L.cg_exchange_state_async(ev.ctx, b, p(ho), p(hi), hi.numel()))

    exchange_all()  # untimed warm-up: allocates the staging buffers
    ev.synchronize()
    barrier()
    torch.cuda.synchronize()
    q0, q1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    q0.record(stream)
    for b, h in enumerate(h_in):
        ev._check(L.cg_upload_state_async(ev.ctx, b, p(h), h.numel()))
    ev.step(1)
    for _ in range(a.e2e_steps - 1):
        # the next step's inputs come in while this step runs, and this step's
        # results go out while the next one runs
        exchange_all()
        ev.step(1)
    for b, h in enumerate(h_out):
        ev._check(L.cg_download_state_async(ev.ctx, b, ctypes.cast(h.data_ptr(), dp), h.numel()))
    q1.record(stream)
    torch.cuda.synchronize()
    ev.synchronize()
    e2e_ms = max_over_ranks(q0.elapsed_time(q1))
    state_bytes = sum(h.numel() * 8 for h in h_in)
    ev.close()
    variants = {}
    for name, opts in (("per_box_launches", {"batch": 0}), ("graph", {"graph": 1})):
        evv, vms = timed(opts, a.steps)
        evv.close()
        variants[name] = {"value": all_pts * a.steps / (vms / 1e3), "ms_per_step": vms / a.steps}
    acc_all = ensemble.gather(acc, world)
    cpu = None
    if rank == 0 and a.cpu_baseline:
        try:
            cpu = cpu_baseline(ensemble.initial_states([specs[16]], order=4, gpu=True)[0], 4)
        except Exception as exc:  # reported, not fatal
            cpu = {"value": None, "error": str(exc)[:200]}
    if rank != 0:
        return
    peak, peak_kind = measured_peaks()
    ms_step = ms / a.steps
    achieved = ALGO_BYTES_MIXED_DUST * all_pts / world / (ms_step / 1e3) / 1e9
    line = {
        "metric": "grid-pt RK4 updates/s (BSSN+dust)", "value": value, "unit": "grid-pt RK4 updates/s",
        "n_gpus": world, "steps": a.steps, "warmup": a.warmup, "ms_per_step": ms_step,
        "higher_is_better": True, "scaling": "strong", "vs_baseline": None, "dtype": "f32+f64",
        "data": "synthetic",
        "config": ensemble_config(specs, world),
        "groups": groups,
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                     "traffic": None, "peak_kind": peak_kind, "algorithmic_bytes_per_update": ALGO_BYTES_MIXED_DUST},
        "e2e": {"value": all_pts * a.e2e_steps / (e2e_ms / 1e3), "unit": "grid-pt RK4 updates/s",
                "h2d_bytes_per_step": state_bytes * world, "d2h_bytes_per_step": state_bytes * world,
                "steps": a.e2e_steps},
        "gpu_launches": 4 * a.steps * max(1, len(groups)),
        "variants": variants,
        "accuracy_vs_fp64": {
            "max_field_err_rel_perturbation": max(v["field_err_rel_perturbation"] for v in acc_all.values()),
            "max_H_ratio": max(v["H_ratio"] for v in acc_all.values()),
            "min_H_ratio": min(v["H_ratio"] for v in acc_all.values()),
            "boxes": len(acc_all)},
        "clocks": clk.summary(),
        "cpu_baseline": cpu,
    }
    print(json.dumps(line))


def run_slab(a, world, rank, local):
    """One box of (n*world) x n x n points cut into `world` x-slabs, one per
    rank, ghost planes exchanged before every substep (NCCL point-to-point;
    on one GPU the periodic self-exchange).  The box is the n^3 GRF box
    repeated along x, so every slab starts from the same n^3 state with its
    own periodic planes as ghosts, as the undivided box would give it."""
    import torch
    import torch.distributed as dist

    from cosmograph_b200 import slab
    from cosmograph_b200.evolution import BoxConfig

    n, g = a.n, slab.ghost_width(a.order)
    mine = slab.split(make_state(n, seed=1, order=a.order), 1, g)[0]
    halo = slab.DistHalo(g) if world > 1 else None
    cfg = BoxConfig(order=a.order, lapse="Harmonic", precision=a.precision)
    se = slab.SlabEvolution([mine], cfg, g, halo=halo)  # one rank: its own periodic planes as ghosts
    for _ in range(max(a.warmup, 0)):
        se.step(1)
    se.ev.synchronize()
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with ClockSampler(local) as clk:
        e0.record(se.stream)
        se.step(a.steps)
        e1.record(se.stream)
        torch.cuda.synchronize()
    se.ev.synchronize()
    ms = e0.elapsed_time(e1)
    if world > 1:
        t = torch.tensor([ms], dtype=torch.float64, device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms = float(t.item())
    pts = n ** 3
    value = world * pts * a.steps / (ms / 1e3)
    peak, peak_kind = measured_peaks()
    achieved = algo_bytes(a.precision) * pts / 4 / (ms / a.steps / 4 / 1e3) / 1e9
    se.close()
    if rank == 0:
        print(json.dumps({
            "metric": "grid-pt RK4 updates/s (BSSN+dust)", "value": value, "unit": "grid-pt RK4 updates/s",
            "n_gpus": world, "steps": a.steps, "warmup": a.warmup, "ms_per_step": ms / a.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic",
            "config": {"workload": f"bssn_dust_{n * world}x{n}x{n}_o{a.order}_xslabs", "slab_planes": n,
                       "ghost_planes": g, "stencil_order": a.order, "lapse": "Harmonic",
                       "precision": a.precision, "parallelism": f"x-slabs x{world}, ghost exchange per substep",
                       "l2": "inputs larger than L2"},
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": achieved / peak, "traffic": None, "peak_kind": peak_kind},
            "e2e": None, "gpu_launches": 4 * a.steps, "clocks": clk.summary(), "cpu_baseline": None,
        }))


def run_reference_arm(a, world, rank):
    """--impl reference: the reference's CPU implementation (oracle/_ref) of the
    same workload, all host threads, rank 0 only."""
    if rank != 0:
        return
    from oracle import build_ref

    n, order = a.n, a.order
    if a.workload == "ensemble":
        # the reference runs one box per process: one 64^3 box of the ensemble
        from cosmograph_b200 import ensemble

        spec = ensemble.standard_ensemble()[16]
        n, order = spec.n, 4
    binp = build_ref.binary_path(n, n, n, order, "fast")
    base = {"metric": "grid-pt RK4 updates/s (BSSN+dust)", "impl": "reference"}
    if not binp.exists():
        print(json.dumps({"impl": "reference", "unavailable": f"{binp.name} was not built"}))
        return
    if a.workload == "ensemble":
        st = ensemble.initial_states([spec], order=4, gpu=False)[0]
    else:
        st = make_state(n, seed=1, order=order, gpu=False)
    threads = os.cpu_count() or 1
    # each step is a full RK4 step of the same box; cap the count so the run
    # stays within a few minutes on the host cores
    with tempfile.TemporaryDirectory(prefix="cg_bench_ref_") as tmp:
        tmp = Path(tmp)
        (tmp / "config.txt").write_text("lapse = Harmonic\n")
        st.save(tmp / "in.bin")
        env = dict(os.environ, OMP_NUM_THREADS=str(threads))
        warm = max(1, min(a.warmup, 1))
        probe = subprocess.run([str(binp), "evolve", str(tmp / "config.txt"), str(tmp / "in.bin"),
                                str(tmp / "out.bin"), str(warm)], capture_output=True, text=True, env=env,
                               timeout=1800)
        t1 = [float(l.split()[2]) for l in probe.stdout.splitlines() if l.startswith("CGSTEP")]
        per = max(t1) if t1 else 60.0
        k = max(1, min(a.steps, int(150.0 / per)))
        proc = subprocess.run([str(binp), "evolve", str(tmp / "config.txt"), str(tmp / "in.bin"),
                               str(tmp / "out.bin"), str(k)], capture_output=True, text=True, env=env,
                              timeout=3600)
    step_s = [float(l.split()[2]) for l in proc.stdout.splitlines() if l.startswith("CGSTEP")]
    if proc.returncode != 0 or not step_s:
        print(json.dumps({"impl": "reference", "unavailable": f"reference run failed: {proc.stderr[-300:]}"}))
        return
    tot = sum(step_s)
    rate = n ** 3 * len(step_s) / tot
    line = dict(base, value=rate, unit="grid-pt RK4 updates/s", n_gpus=a.gpus, steps=len(step_s),
                warmup=warm, ms_per_step=1e3 * tot / len(step_s), higher_is_better=True, scaling="weak",
                vs_baseline=None, dtype="f64", data="synthetic",
                config=(box_config(n, order, a.precision, world) if a.workload != "ensemble" else
                        ensemble_config(ensemble.standard_ensemble(), world)),
                cpu_baseline={"value": rate, "unit": "grid-pt RK4 updates/s", "cores": threads,
                              "kind": "reference",
                              "sample": f"{len(step_s)} RK4 steps (of {a.steps} requested) of one "
                                        f"{n}^3 box; reference sources, {binp.name}"},
                e2e={"value": rate, "unit": "grid-pt RK4 updates/s", "h2d_bytes_per_step": 0,
                     "d2h_bytes_per_step": 0})
    print(json.dumps(line))


def main():
    a = parse()
    world, rank, local = dist_setup(a) if a.impl == "ours" else (
        int(os.environ.get("WORLD_SIZE", "1")), int(os.environ.get("RANK", "0")), 0)
    if a.impl == "reference":
        return run_reference_arm(a, world, rank)
    if a.workload in ("ensemble", "slab"):
        (run_ensemble if a.workload == "ensemble" else run_slab)(a, world, rank, local)
        if world > 1:
            import torch.distributed as dist

            dist.destroy_process_group()
        return

    import torch
    import torch.distributed as dist

    from cosmograph_b200.evolution import BoxConfig, Evolution

    n = a.n
    st = make_state(n, seed=1 + rank, order=a.order)
    cfg = BoxConfig(order=a.order, lapse="Harmonic", precision=a.precision)
    stream = torch.cuda.Stream()
    ev = Evolution(st, cfg)
    ev.set_stream(stream.cuda_stream)
    pts = n ** 3
    launches_per_step = 4

    def barrier():
        if world > 1:
            dist.barrier()

    def max_over_ranks(x):
        if world == 1:
            return x
        t = torch.tensor([x], dtype=torch.float64, device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        return float(t.item())

    # warm-up
    for _ in range(max(a.warmup, 0)):
        ev.step(1)
    ev.synchronize()
    torch.cuda.synchronize()

    # timed: device-resident state
    barrier()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with ClockSampler(local) as clk:
        e0.record(stream)
        for _ in range(a.steps):
            ev.step(1)
        e1.record(stream)
        torch.cuda.synchronize()
    ev.synchronize()
    barrier()
    ms = max_over_ranks(e0.elapsed_time(e1))
    ms_per_step = ms / a.steps
    value = world * pts * a.steps / (ms / 1e3)

    if a.ncu:
        if rank == 0:
            print(json.dumps({"ncu_run": True, "ms_per_step": ms_per_step}))
        ev.close()
        return

    # FP64 state and constraints after warm-up + timed steps (accuracy reference)
    ref_state = ev.download(0) if a.precision == "fp64" else None
    ref_h = ev.constraints(0) if a.precision == "fp64" else None
    peak, peak_kind = measured_peaks()

    # the other arithmetic variants of the same kernel, same workload
    variants = {}
    for prec in [v for v in a.variants.split(",") if v and v != a.precision]:
        ev_v = Evolution(st, BoxConfig(order=a.order, lapse="Harmonic", precision=prec))
        ev_v.set_stream(stream.cuda_stream)
        for _ in range(max(a.warmup, 0)):
            ev_v.step(1)
        ev_v.synchronize()
        barrier()
        torch.cuda.synchronize()
        v0, v1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        v0.record(stream)
        for _ in range(a.steps):
            ev_v.step(1)
        v1.record(stream)
        torch.cuda.synchronize()
        ev_v.synchronize()
        vms = max_over_ranks(v0.elapsed_time(v1))
        vms_step = vms / a.steps
        v_ach = algo_bytes(prec) * pts / launches_per_step / (vms_step / launches_per_step / 1e3) / 1e9
        variants[prec] = {"value": world * pts * a.steps / (vms / 1e3), "ms_per_step": vms_step,
                          "speedup_vs_fp64": ms_per_step / vms_step if a.precision == "fp64" else None,
                          "roofline": {"achieved": v_ach, "peak": peak, "unit": "GB/s", "frac": v_ach / peak,
                                       "algorithmic_bytes_per_update": algo_bytes(prec),
                                       "traffic": profiled_traffic(n, a.order, prec)}}
        if ref_state is not None:
            variants[prec]["accuracy_vs_fp64"] = accuracy(ref_state, ev_v.download(0), ref_h, ev_v.constraints(0))
        ev_v.close()
    del ref_state
    if a.ensemble:
        variants["ensemble"] = ensemble_variant(a, world, rank, stream)
    if a.scalar:
        variants["scalar"] = scalar_variant(a, world, rank, stream)

    # end to end through the C ABI: pinned host state in, one RK4 step, state out
    state_bytes = st.fields.nbytes
    h_in = torch.from_numpy(st.fields.reshape(-1)).pin_memory()
    h_out = torch.empty_like(h_in).pin_memory()
    L = ev.L
    import ctypes

    dp = ctypes.POINTER(ctypes.c_double)
    pin = ctypes.cast(h_in.data_ptr(), dp)
    pout = ctypes.cast(h_out.data_ptr(), dp)
    cnt = h_in.numel()
    # untimed warm-up: the first staged exchange allocates the staging buffers
    ev._check(L.cg_prefetch_state_async(ev.ctx, 0, pin, cnt))
    ev._check(L.cg_exchange_state_async(ev.ctx, 0, pout, pin, cnt))
    ev.synchronize()
    barrier()
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    q0, q1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    q0.record(stream)
    ev._check(L.cg_upload_state_async(ev.ctx, 0, pin, cnt))
    ev.step(1)
    for _ in range(a.e2e_steps - 1):
        # the next step's input comes in while this step runs, and this
        # step's result goes out while the next one runs
        ev._check(L.cg_prefetch_state_async(ev.ctx, 0, pin, cnt))
        ev._check(L.cg_exchange_state_async(ev.ctx, 0, pout, pin, cnt))
        ev.step(1)
    ev._check(L.cg_download_state_async(ev.ctx, 0, pout, cnt))
    q1.record(stream)
    torch.cuda.synchronize()
    ev.synchronize()
    e2e_ms = max_over_ranks(q0.elapsed_time(q1))
    e2e_wall = max_over_ranks(time.perf_counter() - t0)
    e2e_value = world * pts * a.e2e_steps / (e2e_ms / 1e3)
    ev.close()

    algo = algo_bytes(a.precision) * pts / launches_per_step
    launch_ms = ms_per_step / launches_per_step
    achieved = algo / (launch_ms / 1e3) / 1e9
    traffic = profiled_traffic(n, a.order, a.precision)
    # the compute roofline beside the HBM one: counted FP64 flops per update
    # against the measured FP64 peak of this GPU
    compute = None
    flops_upd, fpk = profiled_flops(a.precision), fp64_peak(L)
    if flops_upd and fpk:
        ach_f = flops_upd * pts / (ms_per_step / 1e3)
        compute = {"bound": "fp64", "achieved": ach_f / 1e12, "peak": fpk / 1e12, "unit": "TFLOP/s",
                   "frac": ach_f / fpk, "flops_per_update": flops_upd,
                   "peak_kind": "measured (cg_fp64_peak: FMA chains, CUDA events)"}

    cpu = None
    if rank == 0 and a.cpu_baseline:
        try:
            cpu = cpu_baseline(st, a.order)
        except Exception as exc:  # reported, not fatal
            cpu = {"value": None, "error": str(exc)[:200]}

    if rank == 0:
        line = {
            "metric": "grid-pt RK4 updates/s (BSSN+dust)",
            "value": value,
            "unit": "grid-pt RK4 updates/s",
            "n_gpus": world,
            "steps": a.steps,
            "warmup": a.warmup,
            "ms_per_step": ms_per_step,
            "higher_is_better": True,
            "scaling": "weak",
            "vs_baseline": None,
            "dtype": "f64",
            "data": "synthetic",
            "config": box_config(n, a.order, a.precision, world),
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": achieved / peak, "traffic": traffic, "peak_kind": peak_kind,
                         "algorithmic_bytes_per_launch": algo, "compute": compute},
            "e2e": {"value": e2e_value, "unit": "grid-pt RK4 updates/s",
                    "h2d_bytes_per_step": state_bytes, "d2h_bytes_per_step": state_bytes,
                    "steps": a.e2e_steps, "wall_s": e2e_wall},
            "gpu_launches": launches_per_step * a.steps,
            "variants": variants,
            "clocks": clk.summary(),
            "cpu_baseline": cpu,
        }
        print(json.dumps(line))
    if world > 1:
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
