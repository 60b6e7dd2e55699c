#!/usr/bin/env python
"""Benchmark of the Potts primal-dual segmentation solve on B200.

Workload (one "step" = one full solve): the 768 x 768 x 1024 cylindrical core
(radius 370, 440,434,688 in-mask voxels), K = 3 labels, lambda = 30,
tau = tau' = 1/sqrt(12), 1000 iterations, FP64 energies every 50 iterations.
Input: a seeded synthetic phantom (glass matrix, brine/scCO2 spheres of radius
6-30, Gaussian blur sigma 1, noise 7e-3), generated on the GPU; the state
(~30 GB) is far larger than L2, so no L2 flush is needed between steps.

Metric: in-mask voxel-iterations per second (Gvox-iter/s), whole job.
  value  device-resident input, CUDA events around K solves on the solver's stream
  e2e    the same solves through the host-buffer C-ABI call (pinned u in,
         ci[argmax] + label bytes out), copies inside the timed region
Also: the roofline of the dominant kernel (the fused iteration) from the
solver's own per-iteration device timing, a CPU baseline (the FP64 oracle on
this machine's cores, bounded sample), and "storage": one solve each of the
FP32 split (plain) form and of the bfloat16 / binary16 storage forms on the
same input, with their speed and their label flips and V error against the
FP32 solve (bit-identical to the FP32 plain form).

--workload config2 runs the same volume with K = 4 (a fourth phase at
4.6e-2 on 15% of the pores).  --workload config3 is the batched sweep: 48
sub-volumes with sides drawn from 64..256 per axis, each with its own lambda
and noise, K = 3, 400 iterations, one potts_batch (captured graphs, one
fused launch per iteration over all volumes, autotuned tile); under torchrun
the volumes are bin-packed over the ranks (longest first).  --workload config4
is the differentiable solve: 192^3, r = 90, K = 3, 200 unrolled iterations,
checkpoints every 20, cross-entropy of V against the true labels; value =
voxel-iterations of forward + backward per second; the gradients of c, lambda
and --fd-coords random u coordinates are checked against FP64 central
differences of the FP64 GPU solve (the same bits as the FP64 oracle; step 1e-6
relative, also 1e-4 for u).

--workload tv is TV-L2 denoising (chambolle(), 768^2 x 1024, 150 iterations).
--workload fieldio is the field I/O around the solve on the same core: the
.bin archive of an FP32 field saved and loaded, a uint16 scan's
find_intensity_range + convert_to_fp, and the --rawout VTK label box; value =
in-mask voxels per second through those five kernels, e2e = the same through
host bytes.  --workload labels times the label-finding inputs (min_max,
grad_magn, calc_hist, uv_hist) on the same core.  tvmid / fieldiomid /
labelsmid / mid / mid4 are 384^2 x 256 profiling sizes.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
Under torchrun each rank solves its own phantom (weak scaling, no data-path
collective: the ranks' volumes are independent).
"""
from __future__ import annotations

import argparse
import datetime
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time
from pathlib import Path

ROOT = Path(__file__).resolve().parent
if str(ROOT) not in sys.path:
    sys.path.insert(0, str(ROOT))

METRIC = "Potts PD Gvox-iter/s at k=3, %HBM peak; BF16-store vs FP32 at ≤1e-4 label flips"
UNIT = "Gvox-iter/s"
K_LABELS = 3
LAMBDA = 30.0
RADIUS = {"config1": 370.0, "config2": 370.0, "config0": 60.0, "mid": 180.0, "mid4": 180.0, "prof": 246.0}
STORE_BYTES = {"f32": 4, "bf16": 2, "f16": 2}


def parse_args():
    p = argparse.ArgumentParser(description=__doc__, formatter_class=argparse.RawDescriptionHelpFormatter)
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=None,
                   help="timed steps (default 3; 40 for the label-input workloads, whose step is a few ms)")
    p.add_argument("--warmup", type=int, default=3)
    p.add_argument("--impl", choices=["ours", "reference"], default="ours")
    p.add_argument("--iters", type=int, default=1000)
    p.add_argument("--gap-every", type=int, default=50)
    p.add_argument("--variant", choices=["fused", "plain", "voxel"], default="fused",
                   help="voxel: TV workloads only, the per-voxel fused TV kernel")
    p.add_argument("--storage", choices=["f32", "bf16", "f16"], default="f32",
                   help="state storage of the timed solves")
    p.add_argument("--arith", choices=["exact", "fast"], default="fast",
                   help="FP32 arithmetic of the solves: fast (the default: fewer operations, held to the FP64 "
                        "oracle within 1e-5 relative on V) or exact (the reference's operations, bit-identical to "
                        "the FP32 oracle)")
    p.add_argument("--no-storage-compare", action="store_true",
                   help="skip the FP32-plain / BF16 / FP16 comparison solves")
    p.add_argument("--workload", choices=["config1", "config2", "config3", "config4", "config0", "mid", "mid4", "prof", "tv", "tvmid",
                            "fieldio", "fieldiomid", "labels", "labelsmid"],
                   default="config1",
                   help="config1: 768x768x1024 r=370 (the benchmark); config0: 128^3 r=60; "
                        "mid: 384x384x256 r=180 (profiling size, state > L2); "
                        "prof: 512x512x256 r=246 (profiling size with 5 waves of work items, 3.3 GB)")
    p.add_argument("--fd-coords", type=int, default=64,
                   help="config4: random u coordinates checked against FP64 central differences")
    p.add_argument("--shard", action="store_true",
                   help="config1 as one volume split by columns over the ranks (NCCL halo exchange, strong scaling)")
    p.add_argument("--no-e2e", action="store_true")
    p.add_argument("--no-cpu-baseline", action="store_true")
    p.add_argument("--cpu-seconds", type=float, default=15.0, help="budget of the CPU baseline sample")
    p.add_argument("--tile-rows", type=int, default=0, help="fused tile rows (0 = library default)")
    p.add_argument("--tile-slices", type=int, default=0, help="fused tile slices (0 = library default)")
    p.add_argument("--segment", type=int, default=0, help="columns per fused work item (0 = library default)")
    p.add_argument("--tile-vpt", type=int, default=0, help="fused slices per thread (0 = library default)")
    p.add_argument("--persistent", type=int, choices=[0, 1], default=0,
                   help="fused: 1 = the iterations between energy evaluations in one persistent launch, "
                        "0 = one launch per iteration")
    p.add_argument("--prefetch", type=int, default=0,
                   help="fused: planes of L2 prefetch ahead of the load ring (0 = library default, -1 = none)")
    args = p.parse_args()
    if args.steps is None:
        args.steps = 40 if args.workload in ("labels", "labelsmid") else 3
    if args.variant == "voxel" and args.workload not in ("tv", "tvmid"):
        p.error("--variant voxel applies to the TV workloads only")
    return args


def tau_baseline() -> float:
    import numpy as np

    return float(np.float32(1.0) / np.sqrt(np.float32(12.0)))


# ----------------------------------------------------------------------------- distributed plumbing
class Dist:
    def __init__(self):
        self.world = int(os.environ.get("WORLD_SIZE", "1"))
        self.rank = int(os.environ.get("RANK", "0"))
        self.local = int(os.environ.get("LOCAL_RANK", "0"))
        self.pg = False

    def init(self, backend="nccl"):
        import torch
        import torch.distributed as dist

        if self.world > 1 and not self.pg:
            os.environ.setdefault("MASTER_ADDR", "127.0.0.1")
            kw = {"device_id": torch.device("cuda", self.local)} if backend == "nccl" else {}
            dist.init_process_group(backend, timeout=datetime.timedelta(seconds=900), **kw)
            self.pg = True

    def barrier(self):
        if self.pg:
            import torch.distributed as dist

            dist.barrier()

    def reduce(self, x: float, op: str) -> float:
        if not self.pg:
            return x
        import torch
        import torch.distributed as dist

        t = torch.tensor([x], dtype=torch.float64, device=torch.device("cuda", self.local))
        dist.all_reduce(t, op=dist.ReduceOp.MAX if op == "max" else dist.ReduceOp.SUM)
        return float(t.item())

    def close(self):
        if self.pg:
            import torch.distributed as dist

            dist.destroy_process_group()
            self.pg = False


# ----------------------------------------------------------------------------- clocks
class ClockSampler:
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device_index: int):
        self.dev = device_index
        self.proc = None
        self.path = None

    def start(self):
        try:
            fd, self.path = tempfile.mkstemp(suffix=".csv")
            os.close(fd)
            self.fh = open(self.path, "w")
            self.proc = subprocess.Popen(["nvidia-smi", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                                          "-i", str(self.dev), "-lms", "200"], stdout=self.fh,
                                         stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None

    def stop(self) -> dict:
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        self.fh.close()
        sm, mx, reasons, power = [], [], set(), []
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in Path(self.path).read_text().splitlines():
            f = [x.strip() for x in line.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx.append(float(f[2]))
                power.append(float(f[3]))
            except ValueError:
                continue
            for name, val in zip(names, f[5:9]):
                if val.lower() == "active":
                    reasons.add(name)
        os.unlink(self.path)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["no samples"]}
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": max(mx), "reasons": sorted(reasons),
                "samples": len(sm), "power_w_max": max(power) if power else None}


# ----------------------------------------------------------------------------- peaks / traffic
def measured_peaks() -> dict:
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        try:
            d = json.loads(p.read_text())
            return {"hbm_gbs": float(d["hbm_gbs"]), "source": "measured"}
        except Exception:
            pass
    return {"hbm_gbs": 6650.0, "source": "fallback"}


def profiled_traffic(variant: str) -> dict | None:
    """DRAM bytes per voxel-iteration of the dominant kernel from the committed ncu summary."""
    p = ROOT / "profiles" / "traffic.json"
    if not p.exists():
        return None
    try:
        d = json.loads(p.read_text())
        return d.get(variant)
    except Exception:
        return None


def bytes_per_voxel_iter(variant: str, k: int = K_LABELS, storage: str = "f32") -> int:
    """Algorithmic DRAM bytes per in-mask voxel and iteration (state values of
    STORE_BYTES[storage] bytes, u always FP32).
    fused: Xi (3(K-1)) and V (K-1) read and written once, u read once;
    split: dual launch reads Vbar, Xi and writes Xi; primal launch reads Xi, V, u
           and writes V, Vbar."""
    e = STORE_BYTES[storage]
    if variant == "fused":
        return e * 8 * (k - 1) + 4
    return e * 13 * (k - 1) + 4


# ----------------------------------------------------------------------------- CPU baseline (oracle)
def cpu_sample_phantom():
    """The config-1 cross-section and recipe, 16 slices along the axis, built on the CPU.  The
    cylinder mask comes from the oracle's restatement of the mask constructor, so that this
    phantom (used by the CPU baseline and the reference arm) never loads the GPU library."""
    from oracle import oracle
    from segmentctscans_b200.layout import CylinderMapping, get_stride
    from segmentctscans_b200.phantom import make_phantom

    n, rows, cols, r = 16, 768, 768, 370.0
    sr, base, cb, ce, _ = oracle.cylinder_mask(rows, cols, (cols - 1) / 2.0, (rows - 1) / 2.0, r, get_stride(n))
    m = CylinderMapping(n, rows, cols, get_stride(n), cb, ce, sr, base)
    return make_phantom(n, rows, cols, r, seed=0, radius_range=(6.0, 30.0), noise=7e-3, device="cpu", mapping=m)


def run_cpu_oracle(ph, iters: int, threads: int) -> float:
    from oracle import oracle

    oracle.set_threads(threads)
    u = ph.u.numpy().copy()
    tau = tau_baseline()
    t0 = time.perf_counter()
    oracle.solve(ph.mapping, u, ph.ci, LAMBDA, tau, tau, iters, precision="f64", want_state=False)
    return time.perf_counter() - t0


def cpu_baseline(budget_s: float) -> dict:
    ph = cpu_sample_phantom()
    threads = os.cpu_count() or 1
    t1 = run_cpu_oracle(ph, 1, threads)
    iters = max(1, min(200, int(budget_s / max(t1, 1e-3))))
    t = run_cpu_oracle(ph, iters, threads)
    vox = ph.mapping.data_size
    return {"value": vox * iters / t / 1e9, "unit": UNIT, "cores": threads, "kind": "port",
            "sample": f"FP64 oracle, OpenMP {threads} threads: 768x768 cross-section (r=370), 16 slices "
                      f"({vox} in-mask voxels), K=3, {iters} iterations, {t:.1f} s"}


# ----------------------------------------------------------------------------- reference arm
def run_reference(args, dist_: Dist) -> None:
    if dist_.rank != 0:
        return
    ph = cpu_sample_phantom()
    threads = os.cpu_count() or 1
    t1 = run_cpu_oracle(ph, 1, threads)
    iters = max(1, int(min(args.cpu_seconds / 3.0, 20.0) / max(t1, 1e-3)))
    for _ in range(args.warmup):
        run_cpu_oracle(ph, 1, threads)
    times = [run_cpu_oracle(ph, iters, threads) for _ in range(args.steps)]
    vox = ph.mapping.data_size
    total = sum(times)
    value = vox * iters * args.steps / total / 1e9
    out = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1000 * total / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": "potts_k3_768x768_r370_cpu_sample", "rows": 768, "cols": 768, "n_slices": 16,
                   "radius": 370, "k": K_LABELS, "lambda": LAMBDA, "iters_per_step": iters},
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": threads, "kind": "port",
                         "sample": f"the reference has no CPU implementation of this path and cannot be built "
                                   f"here; FP64 oracle port, {threads} threads, {vox} voxels x {iters} iterations "
                                   f"per step"},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(out), flush=True)


# ----------------------------------------------------------------------------- our arm
def run_ours(args, dist_: Dist) -> None:
    import numpy as np
    import torch

    from segmentctscans_b200 import potts
    from segmentctscans_b200.phantom import config0_phantom, config1_phantom, config2_phantom, make_phantom

    if not torch.cuda.is_available():
        raise SystemExit("bench.py needs a CUDA device")
    dev = torch.device("cuda", dist_.local)
    torch.cuda.set_device(dev)
    dist_.init("nccl")

    if args.workload == "config1":
        ph = config1_phantom(seed=dist_.rank, device=dev)
    elif args.workload == "config2":
        ph = config2_phantom(seed=dist_.rank, device=dev)
    elif args.workload == "config0":
        ph = config0_phantom(seed=dist_.rank, device=dev)
    elif args.workload == "prof":
        ph = make_phantom(256, 512, 512, 246.0, seed=dist_.rank, radius_range=(6.0, 30.0), noise=7e-3, device=dev)
    else:
        ph = make_phantom(256, 384, 384, 180.0, seed=dist_.rank, radius_range=(6.0, 30.0), noise=7e-3, device=dev,
                          k=4 if args.workload == "mid4" else 3)
    m, u, ci = ph.mapping, ph.u, ph.ci
    k = len(ci)
    truth = ph.truth
    del ph
    torch.cuda.empty_cache()
    span = m.span
    tau = tau_baseline()
    variant = 0 if args.variant == "fused" else 1
    stream = torch.cuda.current_stream(dev)
    ctx = potts.make_context(dev.index, stream=stream.cuda_stream)
    res = torch.empty(span, dtype=torch.float32, device=dev)
    lab = torch.empty(span, dtype=torch.uint8, device=dev)

    tile_opts = {"tile_rows": args.tile_rows, "tile_slices": args.tile_slices, "segment_cols": args.segment,
                 "tile_vpt": args.tile_vpt, "prefetch": args.prefetch, "arith": args.arith,
                 "persistent": args.persistent}

    def step():
        return potts.solve_device(ctx, m, u.data_ptr(), ci, LAMBDA, tau, tau, args.iters, res_ptr=res.data_ptr(),
                                  labels_ptr=lab.data_ptr(), stats=True, variant=variant,
                                  gap_every=args.gap_every, storage=args.storage, **tile_opts)

    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize(dev)
    dist_.barrier()
    torch.cuda.synchronize(dev)

    clocks = ClockSampler(dev.index)
    clocks.start()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    stats = [step() for _ in range(args.steps)]
    e1.record(stream)
    torch.cuda.synchronize(dev)
    dist_.barrier()
    clk = clocks.stop()
    t_local = e0.elapsed_time(e1) / 1000.0
    t_max = dist_.reduce(t_local, "max")
    vox = m.data_size
    vox_iters_all = dist_.reduce(float(vox) * args.iters * args.steps, "sum")
    value = vox_iters_all / t_max / 1e9

    # roofline of the fused iteration kernel: algorithmic bytes / average launch time
    loop_ms = sum(s.loop_ms for s in stats)
    loop_launches = sum(s.loop_launches for s in stats)
    loop_iters = sum(s.loop_iters for s in stats)
    launch_s = loop_ms / 1000.0 / max(loop_launches, 1)
    iter_s = loop_ms / 1000.0 / max(loop_iters, 1)
    bpv = bytes_per_voxel_iter(args.variant, k, args.storage)
    # bytes of one iteration over its device time (a persistent launch runs many iterations; the
    # split form runs two launches per iteration)
    achieved = bpv * vox / iter_s / 1e9
    peaks = measured_peaks()
    tr = profiled_traffic((args.variant + ("_fast" if args.arith == "fast" else ""))
                          if args.storage == "f32" and k == 3 and args.tile_rows == 0 else None)
    traffic = tr["dram_bytes_per_voxel_iter"] * vox if tr else None
    roofline = {"bound": "hbm", "achieved": round(achieved, 1), "peak": peaks["hbm_gbs"], "unit": "GB/s",
                "frac": round(achieved / peaks["hbm_gbs"], 4), "traffic": traffic,
                "kernel": ("potts::fused_persistent_kernel" if loop_iters > loop_launches else "potts::fused_tiled_kernel")
                if args.variant == "fused" else "potts::dual_kernel+primal_kernel",
                "bytes_per_voxel_iter": bpv, "avg_launch_ms": round(launch_s * 1000, 4),
                "avg_iter_ms": round(iter_s * 1000, 4), "iters_per_launch": round(loop_iters / max(loop_launches, 1), 2),
                "peak_source": f"{peaks['source']} (MEASURED_PEAKS.json hbm_gbs)"}
    # the same time against the unfused per-voxel traffic (Xi, V and Vbar each read and written once,
    # u read once: 2 * 5 (K - 1) stored values + 4 B), the figure the reference's two-kernel
    # structure has to move; frac above stays on the fused form's own bytes
    sb = 2 * 5 * (k - 1) * STORE_BYTES[args.storage] + 4
    roofline["unfused_bytes_per_voxel_iter"] = sb
    roofline["unfused_frac"] = round(sb * vox / iter_s / 1e9 / peaks["hbm_gbs"], 4)

    # quality figures of the last solve
    last = stats[-1]
    gap = last.energy_trace[-1].tolist() if last.energy_trace is not None else None
    lab_in = lab.view(m.n_lines, m.nstride)[:, : m.n_images]
    tru_in = truth.view(m.n_lines, m.nstride)[:, : m.n_images]
    agree = float((lab_in == tru_in).float().mean().item())

    # end to end through the host-buffer C-ABI call
    e2e = None
    if not args.no_e2e:
        hu = torch.empty(span, dtype=torch.float32, pin_memory=True)
        hu.copy_(u.cpu())
        hres = torch.empty(span, dtype=torch.float32, pin_memory=True)
        hlab = torch.empty(span, dtype=torch.uint8, pin_memory=True)
        hu_np, hres_np, hlab_np = hu.numpy(), hres.numpy(), hlab.numpy()

        def e2e_step():
            potts.solve_host(ctx, m, hu_np, ci, LAMBDA, tau, tau, args.iters, res=hres_np, labels=hlab_np,
                             variant=variant, gap_every=args.gap_every, storage=args.storage, **tile_opts)

        e2e_step()  # allocates the context's staging buffers
        torch.cuda.synchronize(dev)
        dist_.barrier()
        f0, f1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        w0 = time.perf_counter()
        f0.record(stream)
        for _ in range(args.steps):
            e2e_step()
        f1.record(stream)
        torch.cuda.synchronize(dev)
        w1 = time.perf_counter()
        te = max(f0.elapsed_time(f1) / 1000.0, 0.0)
        te = dist_.reduce(max(te, w1 - w0), "max")
        same = bool(np.array_equal(hlab_np, lab.cpu().numpy()))
        e2e = {"value": vox_iters_all / te / 1e9, "unit": UNIT, "h2d_bytes_per_step": 4 * span,
               "d2h_bytes_per_step": 5 * span, "matches_device_run": same}

    storage = None
    if not args.no_storage_compare and args.variant == "fused" and args.storage == "f32":
        storage = storage_compare(args, dist_, ctx, m, u, ci, tau, stream, dev, value)

    cpu = None
    if dist_.rank == 0 and dist_.world == 1 and not args.no_cpu_baseline:
        cpu = cpu_baseline(args.cpu_seconds)

    launches = sum(s.total_launches for s in stats)
    if dist_.rank == 0:
        out = {
            "metric": METRIC, "value": round(value, 3), "unit": UNIT, "n_gpus": dist_.world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": round(1000 * t_max / args.steps, 2), "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32" if args.storage == "f32" else f"f32 math, {args.storage} state",
            "data": "synthetic",
            "config": {"workload": f"potts_k{k}_{m.rows}x{m.cols}x{m.n_images}_r{RADIUS[args.workload]:g}",
                       "rows": m.rows, "cols": m.cols, "n": m.n_images, "radius": RADIUS[args.workload],
                       "in_mask_voxels": vox, "k": k, "lambda": LAMBDA, "tau": tau, "iters": args.iters,
                       "gap_every": args.gap_every, "variant": args.variant, "storage": args.storage,
                       "arith": args.arith,
                       "tile": [args.tile_rows, args.tile_slices, args.tile_vpt, args.segment],
                       "prefetch": args.prefetch, "persistent": args.persistent,
                       "parallelism": f"replica x{dist_.world}" if dist_.world > 1 else "single",
                       "l2": "inputs larger than L2 (state ~30 GB per GPU)"},
            "roofline": roofline, "e2e": e2e, "gpu_launches": launches, "clocks": clk, "cpu_baseline": cpu,
            "storage": storage,
            "quality": {"final_sqrt_max_dV2": last.dq_last, "energy_last": gap, "truth_agreement": round(agree, 5)},
        }
        print(json.dumps(out), flush=True)
    ctx.close()
    dist_.close()


def storage_compare(args, dist_: Dist, ctx, m, u, ci, tau, stream, dev, fused_value: float) -> dict:
    """The FP64 solve of the timed volume (FP64 state and arithmetic, the same bits as the FP64 oracle)
    as the yardstick, then one timed solve each of the FP32 split form, the FP32 fused form of this
    line and the 16-bit storage forms: speed, and label flips (off exact FP64 ties) and relative L2 of
    V against the FP64 solve."""
    import torch

    from segmentctscans_b200 import potts

    k = len(ci)
    span, vox = m.span, m.data_size
    lab = torch.empty(span, dtype=torch.uint8, device=dev)
    v = torch.empty((k - 1) * span, dtype=torch.float32, device=dev)

    def in_mask(x, planes=1):
        return x.view(planes, m.n_lines, m.nstride)[:, :, : m.n_images]

    # the FP64 yardstick
    lab64 = torch.empty(span, dtype=torch.uint8, device=dev)
    v64 = torch.empty((k - 1) * span, dtype=torch.float64, device=dev)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    potts.solve_device_f64(ctx, m, u.data_ptr(), ci, LAMBDA, tau, tau, args.iters, labels_ptr=lab64.data_ptr(),
                           V_ptr=v64.data_ptr(), stats=True, gap_every=args.gap_every)
    e1.record(stream)
    torch.cuda.synchronize(dev)
    f64_value = dist_.reduce(float(vox) * args.iters, "sum") / dist_.reduce(e0.elapsed_time(e1) / 1000.0, "max") / 1e9
    vr = in_mask(v64, k - 1)
    full = torch.cat([vr, 1.0 - vr.sum(0, keepdim=True)], 0)
    top2 = torch.topk(full, 2, dim=0).values
    ties = top2[0] == top2[1]
    del full, top2
    lr = in_mask(lab64)
    vr_norm = float(torch.linalg.vector_norm(vr).item())
    n_vox = dist_.reduce(float(vox), "sum")

    def solve(storage, variant, arith, iters):
        return potts.solve_device(ctx, m, u.data_ptr(), ci, LAMBDA, tau, tau, iters, labels_ptr=lab.data_ptr(),
                                  V_ptr=v.data_ptr(), stats=True, variant=variant, gap_every=args.gap_every,
                                  storage=storage, arith=arith, persistent=args.persistent)

    def timed(storage, variant, arith):
        solve(storage, variant, arith, 2)  # allocations, module load
        torch.cuda.synchronize(dev)
        dist_.barrier()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        st = solve(storage, variant, arith, args.iters)
        e1.record(stream)
        torch.cuda.synchronize(dev)
        t = dist_.reduce(e0.elapsed_time(e1) / 1000.0, "max")
        value = dist_.reduce(float(vox) * args.iters, "sum") / t / 1e9
        iter_s = st.loop_ms / 1000.0 / max(st.loop_iters, 1)
        bpv = bytes_per_voxel_iter("fused" if variant == 0 else "plain", k, storage)
        diff = in_mask(lab) != lr
        flips = int(dist_.reduce(float((diff & ~ties).sum().item()), "sum"))
        dv = float(torch.linalg.vector_norm(in_mask(v, k - 1).double() - vr).item())
        return {"value": round(value, 3), "achieved_gbs": round(bpv * vox / iter_s / 1e9, 1),
                "bytes_per_voxel_iter": bpv, "arith": arith, "label_flips_vs_f64": flips,
                "flip_rate_vs_f64": flips / n_vox, "v_rel_l2_vs_f64": dv / max(vr_norm, 1e-300),
                "gap_last": st.energy_trace[-1].tolist() if st.energy_trace is not None else None}

    out = {"reference": "FP64 solve of the same volume on the GPU (FP64 state and arithmetic, split kernels; "
                        "the same bits as the FP64 CPU oracle, tested at 128^3 x 500 iterations); flips exclude "
                        "voxels whose two largest FP64 V are exactly equal",
           "f64": {"value": round(f64_value, 3), "exact_ties": int(ties.sum().item())}}
    out["f32_plain"] = timed("f32", 1, "exact")
    plain_value = out["f32_plain"]["value"]
    out["f32_fused"] = timed("f32", 0, args.arith)
    out["f32_fused"]["timed_line_value"] = round(fused_value, 3)
    if args.arith == "fast":
        out["f32_fused_exact"] = timed("f32", 0, "exact")
    for storage in ("bf16", "f16"):
        r = timed(storage, 0, args.arith)
        r["speedup_vs_f32_plain"] = round(r["value"] / plain_value, 3)
        r["speedup_vs_f32_fused"] = round(r["value"] / fused_value, 3)
        out[storage] = r
    del lab, v, lab64, v64, vr, lr, ties
    torch.cuda.empty_cache()
    return out


def cpu_baseline_batch(specs, budget_s: float) -> dict:
    from oracle import oracle
    from segmentctscans_b200.phantom import batch_phantom

    spec = min(specs, key=lambda s: s.n * s.rows * s.cols)
    ph = batch_phantom(spec, device="cpu")
    threads = os.cpu_count() or 1
    oracle.set_threads(threads)
    u = ph.u.numpy().copy()
    tau = tau_baseline()
    t0 = time.perf_counter()
    oracle.solve(ph.mapping, u, ph.ci, spec.lam, tau, tau, 1, precision="f64", want_state=False)
    t1 = time.perf_counter() - t0
    iters = max(1, min(400, int(budget_s / max(t1, 1e-3))))
    t0 = time.perf_counter()
    oracle.solve(ph.mapping, u, ph.ci, spec.lam, tau, tau, iters, precision="f64", want_state=False)
    t = time.perf_counter() - t0
    vox = ph.mapping.data_size
    return {"value": vox * iters / t / 1e9, "unit": UNIT, "cores": threads, "kind": "port",
            "sample": f"FP64 oracle, OpenMP {threads} threads: the smallest sub-volume of the sweep "
                      f"({spec.n}x{spec.rows}x{spec.cols}, {vox} in-mask voxels), {iters} iterations, {t:.1f} s"}


def run_batch(args, dist_: Dist) -> None:
    """The batched sweep (config 3) through potts_batch."""
    import numpy as np
    import torch

    from segmentctscans_b200 import potts
    from segmentctscans_b200.phantom import batch_phantom, config3_specs

    if not torch.cuda.is_available():
        raise SystemExit("bench.py needs a CUDA device")
    dev = torch.device("cuda", dist_.local)
    torch.cuda.set_device(dev)
    dist_.init("nccl")
    iters = 400 if args.iters == 1000 else args.iters
    specs = config3_specs(48, seed=0)
    # longest-processing-time bin packing of the volumes over the ranks
    est = [s.n * s.rows * s.cols for s in specs]
    loads = [0] * dist_.world
    owner = {}
    for i in sorted(range(len(specs)), key=lambda i: -est[i]):
        r = min(range(dist_.world), key=lambda r: loads[r])
        owner[i] = r
        loads[r] += est[i]
    mine = [i for i in range(len(specs)) if owner[i] == dist_.rank]
    stream = torch.cuda.current_stream(dev)
    ctx = potts.make_context(dev.index, stream=stream.cuda_stream)
    tau = tau_baseline()
    vols, keep = [], []
    for i in mine:
        ph = batch_phantom(specs[i], device=dev)
        m = ph.mapping
        res = torch.empty(m.span, dtype=torch.float32, device=dev)
        lab = torch.empty(m.span, dtype=torch.uint8, device=dev)
        keep.append((ph, res, lab))
        vols.append(potts.BatchVolume(m, ph.u.data_ptr(), ph.ci, specs[i].lam, res.data_ptr(), lab.data_ptr()))
    tile_opts = {"tile_rows": args.tile_rows, "tile_slices": args.tile_slices, "segment_cols": args.segment,
                 "tile_vpt": args.tile_vpt, "prefetch": args.prefetch, "arith": args.arith,
                 "persistent": args.persistent}
    autotune = int(not any(v > 0 for k, v in tile_opts.items() if k != "arith"))
    batch = potts.Batch(ctx, vols, tau, tau, iters, storage=args.storage, autotune=autotune, **tile_opts)
    info = batch.info()
    vox_local = info.voxels
    for _ in range(args.warmup):
        batch.run(stats=False)
    torch.cuda.synchronize(dev)
    dist_.barrier()
    torch.cuda.synchronize(dev)
    clocks = ClockSampler(dev.index)
    clocks.start()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    stats = [batch.run(stats=True) for _ in range(args.steps)]
    e1.record(stream)
    torch.cuda.synchronize(dev)
    dist_.barrier()
    clk = clocks.stop()
    t_max = dist_.reduce(e0.elapsed_time(e1) / 1000.0, "max")
    vox_all = dist_.reduce(float(vox_local), "sum")
    value = vox_all * iters * args.steps / t_max / 1e9

    launch_s = sum(s.loop_ms for s in stats) / 1000.0 / max(sum(s.loop_launches for s in stats), 1)
    iter_s = sum(s.loop_ms for s in stats) / 1000.0 / max(sum(s.loop_iters for s in stats), 1)
    bpv = bytes_per_voxel_iter("fused", 3, args.storage)
    achieved = bpv * vox_local / iter_s / 1e9
    peaks = measured_peaks()
    roofline = {"bound": "hbm", "achieved": round(achieved, 1), "peak": peaks["hbm_gbs"], "unit": "GB/s",
                "frac": round(achieved / peaks["hbm_gbs"], 4), "traffic": None,
                "kernel": "potts::fused_persistent_kernel (every iteration of all volumes in one launch)"
                if all(s.loop_launches == 1 for s in stats)
                else "potts::fused_tiled_kernel (all volumes per launch)", "bytes_per_voxel_iter": bpv,
                "avg_launch_ms": round(launch_s * 1000, 4), "avg_iter_ms": round(iter_s * 1000, 4),
                "peak_source": f"{peaks['source']} (MEASURED_PEAKS.json hbm_gbs)"}

    e2e = None
    if not args.no_e2e:
        hu = [torch.empty(ph.mapping.span, dtype=torch.float32, pin_memory=True) for ph, _, _ in keep]
        for h, (ph, _, _) in zip(hu, keep):
            h.copy_(ph.u.cpu())
        hres = [torch.empty(ph.mapping.span, dtype=torch.float32, pin_memory=True) for ph, _, _ in keep]
        hlab = [torch.empty(ph.mapping.span, dtype=torch.uint8, pin_memory=True) for ph, _, _ in keep]

        def e2e_step():
            for h, (ph, _, _) in zip(hu, keep):
                ph.u.copy_(h, non_blocking=True)
            batch.run(stats=False)
            for hr, hl, (ph, res, lab) in zip(hres, hlab, keep):
                hr.copy_(res, non_blocking=True)
                hl.copy_(lab, non_blocking=True)

        e2e_step()
        torch.cuda.synchronize(dev)
        dist_.barrier()
        f0, f1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        w0 = time.perf_counter()
        f0.record(stream)
        for _ in range(args.steps):
            e2e_step()
        f1.record(stream)
        torch.cuda.synchronize(dev)
        w1 = time.perf_counter()
        te = dist_.reduce(max(f0.elapsed_time(f1) / 1000.0, w1 - w0), "max")
        spans = sum(ph.mapping.span for ph, _, _ in keep)
        same = all(bool(torch.equal(hl, lab.cpu())) for hl, (_, _, lab) in zip(hlab, keep))
        e2e = {"value": vox_all * iters * args.steps / te / 1e9, "unit": UNIT, "h2d_bytes_per_step": 4 * spans,
               "d2h_bytes_per_step": 5 * spans, "matches_device_run": same}

    cpu = None
    if dist_.rank == 0 and dist_.world == 1 and not args.no_cpu_baseline:
        cpu = cpu_baseline_batch(specs, args.cpu_seconds)
    launches = sum(s.total_launches for s in stats)
    if dist_.rank == 0:
        lams = [s.lam for s in specs]
        out = {
            "metric": METRIC, "value": round(value, 3), "unit": UNIT, "n_gpus": dist_.world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": round(1000 * t_max / args.steps, 2), "higher_is_better": True,
            "scaling": "strong", "vs_baseline": None,
            "dtype": "f32" if args.storage == "f32" else f"f32 math, {args.storage} state", "data": "synthetic",
            "config": {"workload": "potts_k3_batch48_sides64-256", "volumes": len(specs),
                       "volumes_this_rank": len(mine), "in_mask_voxels": int(vox_all), "k": 3,
                       "lambda_range": [round(min(lams), 3), round(max(lams), 3)], "tau": tau, "iters": iters,
                       "storage": args.storage, "arith": args.arith, "tile": list(info.tile),
                       "persistent": info.persistent, "autotuned": bool(autotune),
                       "autotune_ms": round(info.autotune_ms, 1), "work_items": info.n_work,
                       "graph_launches": info.graph_launches,
                       "parallelism": f"volumes bin-packed over {dist_.world} ranks" if dist_.world > 1 else "single",
                       "l2": "inputs larger than L2 (state ~8 GB)"},
            "roofline": roofline, "e2e": e2e, "gpu_launches": launches, "clocks": clk, "cpu_baseline": cpu,
            "quality": {"final_sqrt_max_dV2": stats[-1].dq_last},
        }
        print(json.dumps(out), flush=True)
    batch.close()
    ctx.close()
    dist_.close()


def run_adjoint(args, dist_: Dist) -> None:
    """The differentiable solve (config 4) through potts_forward_ckpt / potts_backward."""
    import numpy as np
    import torch

    from segmentctscans_b200 import potts
    from segmentctscans_b200.phantom import make_phantom

    if not torch.cuda.is_available():
        raise SystemExit("bench.py needs a CUDA device")
    dev = torch.device("cuda", dist_.local)
    torch.cuda.set_device(dev)
    dist_.init("nccl")
    iters = 200 if args.iters == 1000 else args.iters
    every, eps, lam = 20, 1e-3, LAMBDA
    tau = tau_baseline()
    ph = make_phantom(192, 192, 192, 90.0, seed=dist_.rank, radius_range=(4.0, 12.0), noise=7e-3, device=dev)
    m, u, ci = ph.mapping, ph.u, ph.ci
    truth = ph.truth
    stream = torch.cuda.current_stream(dev)
    ctx = potts.make_context(dev.index, stream=stream.cuda_stream)
    gu = torch.zeros(m.span, dtype=torch.float32, device=dev)

    def step():
        with potts.Tape(ctx, m, u.data_ptr(), truth.data_ptr(), ci, lam, tau, tau, iters, every, eps) as t:
            gc, gl = t.backward(gu.data_ptr())
            return t.loss, gc, gl

    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize(dev)
    dist_.barrier()
    clocks = ClockSampler(dev.index)
    clocks.start()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    launches0 = potts._native.host_lib().potts_context_launches(ctx.handle)
    e0.record(stream)
    for _ in range(args.steps):
        loss, gc, gl = step()
    e1.record(stream)
    launches = potts._native.host_lib().potts_context_launches(ctx.handle) - launches0
    torch.cuda.synchronize(dev)
    dist_.barrier()
    clk = clocks.stop()
    t_max = dist_.reduce(e0.elapsed_time(e1) / 1000.0, "max")
    vox = m.data_size
    value = dist_.reduce(float(vox) * iters * args.steps, "sum") / t_max / 1e9

    check = None
    if dist_.rank == 0 and args.fd_coords >= 0:
        # FP64 losses through the FP64 GPU solve (the same bits as the FP64 CPU oracle)
        u_h = u.cpu().numpy().copy()
        idx_t = torch.from_numpy(np.arange(m.span).reshape(m.n_lines, m.nstride)[:, : m.n_images].reshape(-1)).to(dev)
        t_in = truth.long()[idx_t].clamp(max=len(ci) - 1)
        V64 = torch.empty((len(ci) - 1, m.span), dtype=torch.float64, device=dev)

        def loss64(uu, cc, ll):
            du = torch.from_numpy(np.ascontiguousarray(uu, np.float32)).to(dev)
            potts.solve_device_f64(ctx, m, du.data_ptr(), cc, ll, tau, tau, iters, V_ptr=V64.data_ptr(), stats=False)
            torch.cuda.synchronize(dev)
            Vm = V64[:, idx_t]
            Vf = torch.cat([Vm, 1.0 - Vm.sum(0, keepdim=True)])
            return float(-torch.log(Vf.gather(0, t_in[None])[0] + eps).mean().item())

        def cd(fun, x, rel):
            h = rel * max(abs(x), 1e-2)
            xp, xm = np.float32(x + h), np.float32(x - h)
            return (fun(float(xp)) - fun(float(xm))) / (float(xp) - float(xm))

        def init_flips(c2):
            # in-mask voxels whose nearest label (the initial state) changes between ci and c2
            a = np.argmin(np.abs(np.asarray(ci, np.float32)[:, None] - u_in[None]), 0)
            b = np.argmin(np.abs(np.asarray(c2, np.float32)[:, None] - u_in[None]), 0)
            return int(np.sum(a != b))

        t0 = time.perf_counter()
        u_in = u_h.reshape(m.n_lines, m.nstride)[:, : m.n_images].reshape(-1)
        rows = []
        for i in range(len(ci)):
            def fc(v, i=i):
                c2 = list(ci)
                c2[i] = v
                return loss64(u_h, c2, lam)
            # the step starts at 1e-6 relative and shrinks while it would move a voxel's nearest
            # label (the initial state is piecewise constant in c: that is a jump, not the derivative)
            def steps(rel):
                h = rel * abs(ci[i])
                return float(np.float32(ci[i] + h)), float(np.float32(ci[i] - h))

            # central where neither side moves a nearest label, else one-sided on the side that moves
            # none (a voxel within FP32 spacing of a tie makes every central step a jump)
            rel, kind, one_sided = 1e-6, "central", None
            while True:
                cp, cm = steps(rel)
                fp = init_flips([cp if k == i else c for k, c in enumerate(ci)])
                fm = init_flips([cm if k == i else c for k, c in enumerate(ci)])
                if fp + fm == 0:
                    g = (fc(cp) - fc(cm)) / (cp - cm)
                    break
                if one_sided is None and fp == 0:
                    one_sided = ("forward", rel, cp)
                elif one_sided is None and fm == 0:
                    one_sided = ("backward", rel, cm)
                nxt = steps(rel / 4.0)
                if nxt[0] == nxt[1]:  # FP32 cannot take a smaller step
                    if one_sided is not None:
                        kind, rel, x1 = one_sided
                        g = (fc(x1) - fc(ci[i])) / (x1 - ci[i])
                    else:
                        rel = 1e-6
                        cp, cm = steps(rel)
                        kind, g = "central (jumps on both sides)", (fc(cp) - fc(cm)) / (cp - cm)
                    break
                rel /= 4.0
            rows.append({"param": f"c{i + 1}", "step": rel, "difference": kind, "adjoint": float(gc[i]),
                         "fd": float(g), "rel": float(abs(gc[i] - g) / abs(g))})
        g = cd(lambda v: loss64(u_h, ci, v), lam, 1e-6)
        rows.append({"param": "lambda", "adjoint": float(gl), "fd": float(g), "rel": float(abs(gl - g) / abs(g))})
        gu_h = gu.cpu().numpy()
        rng = np.random.default_rng(0)
        idx = np.arange(m.span).reshape(m.n_lines, m.nstride)[:, : m.n_images].reshape(-1)
        for j in rng.choice(idx, args.fd_coords, replace=False):
            def fu(v, j=j):
                u2 = u_h.copy()
                u2[j] = v
                return loss64(u2, ci, lam)
            for rel in (1e-6, 1e-4):
                g = cd(fu, float(u_h[j]), rel)
                rows.append({"param": f"u[{int(j)}]", "step": rel, "adjoint": float(gu_h[j]), "fd": float(g),
                             "rel": float(abs(gu_h[j] - g) / abs(g) if g != 0 else abs(gu_h[j]))})
        # scalars: rows whose differences cross a nearest-label tie on both sides measure a jump of
        # the loss (a voxel within FP32 spacing of a tie), not its derivative; they are reported,
        # not held to the tolerance.  u: relative L2 over the sampled coordinates, per step.
        smooth = [r for r in rows[: len(ci) + 1] if "jumps" not in r.get("difference", "")]
        u_l2 = {}
        for step in (1e-6, 1e-4):
            ur = [r for r in rows[len(ci) + 1:] if r["step"] == step]
            a = np.array([r["adjoint"] for r in ur])
            f = np.array([r["fd"] for r in ur])
            u_l2[str(step)] = float(np.linalg.norm(a - f) / max(np.linalg.norm(f), 1e-300))
        check = {"loss_fp64": loss64(u_h, ci, lam), "loss_gpu": float(loss), "fd_step_rel": 1e-6, "rows": rows,
                 "max_rel_scalar": max(r["rel"] for r in smooth) if smooth else None,
                 "scalars_at_label_ties": [r["param"] for r in rows[: len(ci) + 1] if r not in smooth],
                 "u_rel_l2": u_l2, "seconds": time.perf_counter() - t0}

    if dist_.rank == 0:
        out = {
            "metric": METRIC, "value": round(value, 3), "unit": UNIT, "n_gpus": dist_.world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": round(1000 * t_max / args.steps, 2), "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": {"workload": "potts_k3_192x192x192_r90_adjoint", "in_mask_voxels": vox, "k": 3,
                       "lambda": lam, "tau": tau, "iters": iters, "checkpoint_every": every, "loss_eps": eps,
                       "step": "forward with checkpoints + loss + backward (gradients of u, c, lambda)",
                       "parallelism": f"replica x{dist_.world}" if dist_.world > 1 else "single"},
            "roofline": None, "e2e": None, "gpu_launches": launches, "clocks": clk, "cpu_baseline": None,
            "gradient_check": check,
        }
        print(json.dumps(out), flush=True)
    ctx.close()
    dist_.close()


def run_tv(args, dist_: Dist) -> None:
    """TV-L2 denoising (chambolle(), the next row after the Potts solve) on the 768^2 x 1024 core:
    lambda = 0.06, tau = 0.99/6, 150 iterations as totalvarmin.cpp:60,140 calls it."""
    import numpy as np
    import torch

    from segmentctscans_b200 import potts
    from segmentctscans_b200.phantom import config1_phantom

    if not torch.cuda.is_available():
        raise SystemExit("bench.py needs a CUDA device")
    dev = torch.device("cuda", dist_.local)
    torch.cuda.set_device(dev)
    dist_.init("nccl")
    iters = 150 if args.iters == 1000 else args.iters
    lam, tau = 0.06, 0.99 / 6.0
    if args.workload == "tvmid":  # the profiling-size volume
        from segmentctscans_b200.phantom import make_phantom

        ph = make_phantom(256, 384, 384, 180.0, seed=dist_.rank, radius_range=(6.0, 30.0), noise=7e-3, device=dev)
    else:
        ph = config1_phantom(seed=dist_.rank, device=dev)
    m, u = ph.mapping, ph.u
    stream = torch.cuda.current_stream(dev)
    ctx = potts.make_context(dev.index, stream=stream.cuda_stream)
    g = torch.empty_like(u)

    variant = {"fused": 0, "plain": 1, "voxel": 2}[args.variant]

    def step():
        g.copy_(u)
        return potts.tv_denoise(ctx, m, g.data_ptr(), lam, tau, iters, variant=variant)

    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize(dev)
    dist_.barrier()
    clocks = ClockSampler(dev.index)
    clocks.start()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    stats = [step() for _ in range(args.steps)]
    e1.record(stream)
    torch.cuda.synchronize(dev)
    dist_.barrier()
    clk = clocks.stop()
    t_max = dist_.reduce(e0.elapsed_time(e1) / 1000.0, "max")
    vox = m.data_size
    value = dist_.reduce(float(vox) * iters * args.steps, "sum") / t_max / 1e9
    launch_s = sum(s.loop_ms for s in stats) / 1000.0 / max(sum(s.loop_launches for s in stats), 1)
    iter_s = sum(s.loop_ms for s in stats) / 1000.0 / max(sum(s.loop_iters for s in stats), 1)
    # tiled: xi (3) and the differences of g (3) in, xi (3) out; per-voxel fused: xi (3) and g in,
    # xi (3) out; split: div reads xi (3), writes v; grad reads v, g, xi (3), writes xi (3)
    bpv = {0: 36, 1: 48, 2: 28}[variant]
    achieved = bpv * vox / iter_s / 1e9
    peaks = measured_peaks()
    roofline = {"bound": "hbm", "achieved": round(achieved, 1), "peak": peaks["hbm_gbs"], "unit": "GB/s",
                "frac": round(achieved / peaks["hbm_gbs"], 4), "traffic": None,
                "kernel": {0: "potts::tv_tiled_kernel<8,128>", 1: "potts::tv_div_kernel + tv_grad_kernel (average launch)",
                           2: "potts::tv_fused_kernel"}[variant],
                "bytes_per_voxel_iter": bpv,
                "avg_launch_ms": round(launch_s * 1000, 4),
                "peak_source": f"{peaks['source']} (MEASURED_PEAKS.json hbm_gbs)"}
    e2e = None
    if not args.no_e2e:
        hu = torch.empty(m.span, dtype=torch.float32, pin_memory=True)
        hu.copy_(u.cpu())
        hout = torch.empty(m.span, dtype=torch.float32, pin_memory=True)

        def e2e_step():
            g.copy_(hu, non_blocking=True)
            potts.tv_denoise(ctx, m, g.data_ptr(), lam, tau, iters, variant=variant, stats=False)
            hout.copy_(g, non_blocking=True)

        e2e_step()
        torch.cuda.synchronize(dev)
        f0, f1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        w0 = time.perf_counter()
        f0.record(stream)
        for _ in range(args.steps):
            e2e_step()
        f1.record(stream)
        torch.cuda.synchronize(dev)
        te = dist_.reduce(max(f0.elapsed_time(f1) / 1000.0, time.perf_counter() - w0), "max")
        e2e = {"value": dist_.reduce(float(vox) * iters * args.steps, "sum") / te / 1e9, "unit": UNIT,
               "h2d_bytes_per_step": 4 * m.span, "d2h_bytes_per_step": 4 * m.span}
    cpu = None
    if dist_.rank == 0 and dist_.world == 1 and not args.no_cpu_baseline:
        from oracle import oracle

        sph = cpu_sample_phantom()
        threads = os.cpu_count() or 1
        oracle.set_threads(threads)
        su = sph.u.numpy().copy()
        t0 = time.perf_counter()
        oracle.tv(sph.mapping, su, lam, tau, 1, "f64")
        t1 = time.perf_counter() - t0
        # solves of up to 150 iterations (the reference's count), repeated to fill the budget
        it_cpu = max(1, min(150, int(args.cpu_seconds / max(t1, 1e-3))))
        reps, t0 = 0, time.perf_counter()
        while reps == 0 or time.perf_counter() - t0 < args.cpu_seconds:
            oracle.tv(sph.mapping, su, lam, tau, it_cpu, "f64")
            reps += 1
        tc = time.perf_counter() - t0
        cpu = {"value": sph.mapping.data_size * it_cpu * reps / tc / 1e9, "unit": UNIT, "cores": threads,
               "kind": "port",
               "sample": f"FP64 TV oracle, OpenMP {threads} threads: 768x768 cross-section, 16 slices, "
                         f"{reps} solves of {it_cpu} iterations, {tc:.1f} s"}
    if dist_.rank == 0:
        out = {
            "metric": METRIC, "value": round(value, 3), "unit": UNIT, "n_gpus": dist_.world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": round(1000 * t_max / args.steps, 2), "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": {"workload": f"tv_{m.rows}x{m.cols}x{m.n_images}", "in_mask_voxels": vox,
                       "lambda": lam, "tau": tau, "iters": iters, "variant": args.variant,
                       "parallelism": f"replica x{dist_.world}" if dist_.world > 1 else "single",
                       "l2": "inputs larger than L2"},
            "roofline": roofline, "e2e": e2e, "gpu_launches": sum(s.total_launches for s in stats), "clocks": clk,
            "cpu_baseline": cpu, "quality": {"final_sqrt_max_dxi2": stats[-1].dq_last},
        }
        print(json.dumps(out), flush=True)
    ctx.close()
    dist_.close()


def run_fieldio(args, dist_: Dist) -> None:
    """Field I/O around the solve on the 768^2 x 1024 core: the .bin archive of an FP32 field loaded
    (Field<float>::load, the potts-model input) and saved (Field<float>::save, the transpose output),
    a uint16 scan's find_intensity_range + convert_to_fp (transpose), and the --rawout VTK label box
    (potts-model).  value = in-mask voxels per second through the five device kernels of one step;
    e2e = the same step through the C ABI with host (pinned) bytes in and out."""
    import numpy as np
    import torch

    from segmentctscans_b200 import potts
    from segmentctscans_b200.phantom import config1_phantom, make_phantom

    if not torch.cuda.is_available():
        raise SystemExit("bench.py needs a CUDA device")
    dev = torch.device("cuda", dist_.local)
    torch.cuda.set_device(dev)
    dist_.init("nccl")
    if args.workload == "fieldiomid":
        ph = make_phantom(256, 384, 384, 180.0, seed=dist_.rank, radius_range=(6.0, 30.0), noise=7e-3, device=dev)
    else:
        ph = config1_phantom(seed=dist_.rank, device=dev)
    m, u = ph.mapping, ph.u
    vox = m.data_size
    stream = torch.cuda.current_stream(dev)
    ctx = potts.make_context(dev.index, stream=stream.cuda_stream)
    # a uint16 scan of the same phantom (the transpose input) and the output buffers
    w16 = (u * 50000.0 + 1000.0).clamp_(0, 65535).to(torch.int32).to(torch.int16)
    g = torch.empty_like(u)
    un = torch.empty_like(u)
    n_arch, _ = potts.archive_size(m, "f32")
    s, rows, cols, _ = potts.raw_labels_dims(m)
    box_bytes = s * rows * cols
    h_arch = torch.empty(n_arch, dtype=torch.uint8, pin_memory=True)
    h_vtk = torch.empty(box_bytes + 4096, dtype=torch.uint8, pin_memory=True)
    a_np, v_np = h_arch.numpy(), h_vtk.numpy()
    d_box = torch.empty(box_bytes, dtype=torch.uint8, device=dev)

    def step(host: bool):
        """One pass; returns the kernel times (ms) of the five kernels."""
        _, t_save = potts.archive_save(ctx, m, "f32", u.data_ptr(), 0.0, 1.0, out=a_np)
        _, t_load = potts.archive_load(ctx, a_np, "f32", g.data_ptr(), m.span)
        e = [torch.cuda.Event(enable_timing=True) for _ in range(4)]
        e[0].record(stream)
        lo, hi, _ = potts.find_intensity_range(ctx, m, w16.data_ptr(), 1e-4)
        e[1].record(stream)
        potts.convert_to_fp(ctx, m, "u16", w16.data_ptr(), float(lo), float(hi), un.data_ptr())
        e[2].record(stream)
        if host:
            _, t_box = potts.vtk_labels(ctx, m, u.data_ptr(), out=v_np)
        else:
            potts.raw_labels(ctx, m, u.data_ptr(), d_box.data_ptr())
            e[3].record(stream)
        torch.cuda.synchronize(dev)
        t_hist = e[0].elapsed_time(e[1])
        t_conv = e[1].elapsed_time(e[2])
        if not host:
            t_box = e[2].elapsed_time(e[3])
        return {"pack": t_save, "unpack": t_load, "u16_hist": t_hist, "convert_to_fp": t_conv, "raw_box": t_box}

    for _ in range(args.warmup):
        step(False)
    # size-independent check at full size: the archive round trip reproduces every in-mask value
    mv = g.view(m.n_lines, m.nstride)[:, : m.n_images]
    assert torch.equal(mv.view(torch.int32), u.view(m.n_lines, m.nstride)[:, : m.n_images].view(torch.int32))
    torch.cuda.synchronize(dev)
    dist_.barrier()
    clocks = ClockSampler(dev.index)
    clocks.start()
    launches0 = potts._native.host_lib().potts_context_launches(ctx.handle)
    times = [step(False) for _ in range(args.steps)]
    launches = potts._native.host_lib().potts_context_launches(ctx.handle) - launches0
    torch.cuda.synchronize(dev)
    dist_.barrier()
    clk = clocks.stop()
    avg = {k: sum(t[k] for t in times) / len(times) for k in times[0]}
    t_step = sum(avg.values()) / 1000.0
    t_max = dist_.reduce(t_step * args.steps, "max")
    value = dist_.reduce(float(vox) * args.steps, "sum") / t_max / 1e9
    # algorithmic bytes per launch
    algo = {"unpack": 8 * vox, "pack": 8 * vox, "u16_hist": 2 * vox, "convert_to_fp": 6 * vox,
            "raw_box": 4 * vox + box_bytes}
    peaks = measured_peaks()
    kernels = {k: {"avg_ms": round(avg[k], 4), "gbs": round(algo[k] / (avg[k] / 1000.0) / 1e9, 1),
                   "frac": round(algo[k] / (avg[k] / 1000.0) / 1e9 / peaks["hbm_gbs"], 4),
                   "bytes_per_launch": algo[k]} for k in avg}
    roofline = {"bound": "hbm", "achieved": kernels["unpack"]["gbs"], "peak": peaks["hbm_gbs"], "unit": "GB/s",
                "frac": kernels["unpack"]["frac"], "traffic": None, "kernel": "potts::archive_unpack_kernel<32>",
                "bytes_per_voxel": 8, "avg_launch_ms": kernels["unpack"]["avg_ms"],
                "peak_source": f"{peaks['source']} (MEASURED_PEAKS.json hbm_gbs)"}
    e2e = None
    if not args.no_e2e:
        f0, f1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        w0 = time.perf_counter()
        f0.record(stream)
        for _ in range(args.steps):
            step(True)
        f1.record(stream)
        torch.cuda.synchronize(dev)
        te = dist_.reduce(max(f0.elapsed_time(f1) / 1000.0, time.perf_counter() - w0), "max")
        e2e = {"value": dist_.reduce(float(vox) * args.steps, "sum") / te / 1e9, "unit": "Gvox/s",
               "h2d_bytes_per_step": n_arch, "d2h_bytes_per_step": n_arch + box_bytes,
               "note": "archive saved to and loaded from pinned host bytes, VTK file assembled in pinned host memory"}
    cpu = None
    if dist_.rank == 0 and dist_.world == 1 and not args.no_cpu_baseline:
        from oracle import oracle

        sph = cpu_sample_phantom()
        su = sph.u.numpy().copy()
        data, _ = oracle.archive_encode(sph.mapping, su, "f32", 0.0, 1.0)
        reps, t0 = 0, time.perf_counter()
        while reps == 0 or time.perf_counter() - t0 < min(args.cpu_seconds, 15.0):
            oracle.archive_decode(data, "f32")
            oracle.archive_encode(sph.mapping, su, "f32", 0.0, 1.0)
            reps += 1
        tc = time.perf_counter() - t0
        cpu = {"value": sph.mapping.data_size * reps / (tc / 2.0) / 1e9, "unit": "Gvox/s", "cores": 1, "kind": "port",
               "sample": f"bit-serial C oracle, 1 thread: archive decode + encode of the 768x768 cross-section, "
                         f"16 slices ({sph.mapping.data_size} voxels), {reps} rounds in {tc:.1f} s; value per pass"}
    if dist_.rank == 0:
        out = {
            "metric": "field I/O Gvox/s (archive load + save, intensity range + convert_to_fp, raw label box)",
            "value": round(value, 3), "unit": "Gvox/s", "n_gpus": dist_.world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": round(1000 * t_max / args.steps, 3), "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "u8", "data": "synthetic",
            "config": {"workload": f"fieldio_{m.rows}x{m.cols}x{m.n_images}", "in_mask_voxels": vox,
                       "archive_bytes": n_arch, "box_bytes": box_bytes,
                       "parallelism": f"replica x{dist_.world}" if dist_.world > 1 else "single",
                       "l2": "inputs larger than L2"},
            "roofline": roofline, "kernels": kernels, "e2e": e2e, "gpu_launches": launches, "clocks": clk,
            "cpu_baseline": cpu, "check": "archive round trip equal on every in-mask voxel",
        }
        print(json.dumps(out), flush=True)
    ctx.close()
    dist_.close()


def run_labels(args, dist_: Dist) -> None:
    """Label-finding inputs (the GPU steps before the solve: min_max, grad_magn, calc_hist, uv_hist)
    on the 768^2 x 1024 core.  value = in-mask voxels per second through the four calls of one step;
    each call's device time (CUDA events around it on the context's stream, including its small
    result copy) against its algorithmic bytes."""
    import torch

    from segmentctscans_b200 import potts
    from segmentctscans_b200.phantom import config1_phantom, make_phantom

    if not torch.cuda.is_available():
        raise SystemExit("bench.py needs a CUDA device")
    dev = torch.device("cuda", dist_.local)
    torch.cuda.set_device(dev)
    dist_.init("nccl")
    if args.workload == "labelsmid":
        ph = make_phantom(256, 384, 384, 180.0, seed=dist_.rank, radius_range=(6.0, 30.0), noise=7e-3, device=dev)
    else:
        ph = config1_phantom(seed=dist_.rank, device=dev)
    m, u = ph.mapping, ph.u
    vox = m.data_size
    stream = torch.cuda.current_stream(dev)
    ctx = potts.make_context(dev.index, stream=stream.cuda_stream)
    v = torch.empty_like(u)

    def step():
        e = [torch.cuda.Event(enable_timing=True) for _ in range(5)]
        e[0].record(stream)
        potts.min_max(ctx, m, u.data_ptr())
        e[1].record(stream)
        potts.grad_magn(ctx, m, u.data_ptr(), v.data_ptr())
        e[2].record(stream)
        potts.calc_hist_auto(ctx, m, u.data_ptr(), 1024)
        e[3].record(stream)
        potts.uv_hist_auto(ctx, m, u.data_ptr(), v.data_ptr(), 512)
        e[4].record(stream)
        torch.cuda.synchronize(dev)
        return {k: e[i].elapsed_time(e[i + 1]) for i, k in enumerate(("min_max", "grad_magn", "calc_hist_auto",
                                                                          "uv_hist_auto"))}

    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize(dev)
    dist_.barrier()
    clocks = ClockSampler(dev.index)
    clocks.start()
    launches0 = potts._native.host_lib().potts_context_launches(ctx.handle)
    times = [step() for _ in range(args.steps)]
    launches = potts._native.host_lib().potts_context_launches(ctx.handle) - launches0
    torch.cuda.synchronize(dev)
    dist_.barrier()
    clk = clocks.stop()
    avg = {k: sum(t[k] for t in times) / len(times) for k in times[0]}
    t_max = dist_.reduce(sum(avg.values()) / 1000.0 * args.steps, "max")
    value = dist_.reduce(float(vox) * args.steps, "sum") / t_max / 1e9
    # algorithmic bytes per call: min_max reads u; grad_magn reads u (neighbours from cache) and
    # writes v; calc_hist_auto = min_max + histogram, two reads of u; uv_hist_auto = the min/max of v
    # and of u, then the histogram of (u, v): reads v, u, then u and v
    algo = {"min_max": 4 * vox, "grad_magn": 8 * vox, "calc_hist_auto": 8 * vox, "uv_hist_auto": 16 * vox}
    peaks = measured_peaks()
    kernels = {k: {"avg_ms": round(avg[k], 4), "gbs": round(algo[k] / (avg[k] / 1000.0) / 1e9, 1),
                   "frac": round(algo[k] / (avg[k] / 1000.0) / 1e9 / peaks["hbm_gbs"], 4),
                   "bytes_per_call": algo[k]} for k in avg}
    # the dominant call: uv_hist_auto (its ranges in one pass over u and v, the coarse cell count
    # over every 8th line, the hot-cell histogram), against its 16 B per voxel
    roofline = {"bound": "hbm", "achieved": kernels["uv_hist_auto"]["gbs"], "peak": peaks["hbm_gbs"], "unit": "GB/s",
                "frac": kernels["uv_hist_auto"]["frac"], "traffic": None,
                "kernel": "uv_hist_auto: potts::minmax_pair_partial_kernel, potts::uv_coarse_kernel, "
                          "potts::uv_hist_hot_kernel",
                "bytes_per_voxel": 16, "avg_launch_ms": kernels["uv_hist_auto"]["avg_ms"],
                "peak_source": f"{peaks['source']} (MEASURED_PEAKS.json hbm_gbs)"}
    e2e = None
    if not args.no_e2e:
        hu = torch.empty(m.span, dtype=torch.float32, pin_memory=True)
        hu.copy_(u.cpu())
        d_in = torch.empty_like(u)

        def e2e_step():
            d_in.copy_(hu, non_blocking=True)
            potts.min_max(ctx, m, d_in.data_ptr())
            potts.grad_magn(ctx, m, d_in.data_ptr(), v.data_ptr())
            potts.calc_hist_auto(ctx, m, d_in.data_ptr(), 1024)
            potts.uv_hist_auto(ctx, m, d_in.data_ptr(), v.data_ptr(), 512)

        e2e_step()
        torch.cuda.synchronize(dev)
        w0 = time.perf_counter()
        for _ in range(args.steps):
            e2e_step()
        torch.cuda.synchronize(dev)
        te = dist_.reduce(time.perf_counter() - w0, "max")
        e2e = {"value": dist_.reduce(float(vox) * args.steps, "sum") / te / 1e9, "unit": "Gvox/s",
               "h2d_bytes_per_step": 4 * m.span,
               "d2h_bytes_per_step": 8 + (8 + 4 * 1024) + (16 + 4 * potts._native.host_lib().potts_uv_hist_span(512)),
               "note": "u copied in from pinned host memory each step; results (ranges, histograms) read back"}
    cpu = None
    if dist_.rank == 0 and dist_.world == 1 and not args.no_cpu_baseline:
        from oracle import oracle

        sph = cpu_sample_phantom()
        su = sph.u.numpy().copy()
        reps, t0 = 0, time.perf_counter()
        while reps == 0 or time.perf_counter() - t0 < min(args.cpu_seconds, 15.0):
            lo, hi = oracle.min_max(sph.mapping, su)
            sv = oracle.grad_magn(sph.mapping, su)
            oracle.calc_hist(sph.mapping, su, lo, hi, 1024)
            vs, ve = oracle.min_max(sph.mapping, sv, positive=True)
            oracle.uv_hist(sph.mapping, su, sv, lo, hi, vs, ve, 512)
            reps += 1
        tc = time.perf_counter() - t0
        cpu = {"value": sph.mapping.data_size * reps / tc / 1e9, "unit": "Gvox/s", "cores": 1, "kind": "port",
               "sample": f"C oracle, 1 thread: min_max, grad_magn, calc_hist, uv_hist of the 768x768 cross-section, "
                         f"16 slices ({sph.mapping.data_size} voxels), {reps} rounds in {tc:.1f} s"}
    if dist_.rank == 0:
        out = {
            "metric": "label-finding inputs Gvox/s (min_max, grad_magn, calc_hist 1024 bins, uv_hist 512x512)",
            "value": round(value, 3), "unit": "Gvox/s", "n_gpus": dist_.world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": round(1000 * t_max / args.steps, 3), "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": {"workload": f"labels_{m.rows}x{m.cols}x{m.n_images}", "in_mask_voxels": vox,
                       "parallelism": f"replica x{dist_.world}" if dist_.world > 1 else "single",
                       "l2": "inputs larger than L2"},
            "roofline": roofline, "kernels": kernels, "e2e": e2e, "gpu_launches": launches, "clocks": clk,
            "cpu_baseline": cpu,
        }
        print(json.dumps(out), flush=True)
    ctx.close()
    dist_.close()


def run_shard(args, dist_: Dist) -> None:
    """One volume (768 x 768 x 1024, r = 370, K = 3) split by columns over the ranks, one shard per
    GPU, halos over NCCL (potts_shard_*): strong scaling, value = the volume's voxel-iterations per
    second over the slowest rank's device time."""
    import torch

    from segmentctscans_b200 import potts
    from segmentctscans_b200.phantom import config1_phantom
    from segmentctscans_b200.sharding import Shard, destroy_comm, native_bounds, native_cuts, nccl_comm, run_shards

    if not torch.cuda.is_available():
        raise SystemExit("bench.py needs a CUDA device")
    dev = torch.device("cuda", dist_.local)
    torch.cuda.set_device(dev)
    dist_.init("nccl")
    ph = config1_phantom(seed=0, device=dev)  # the same volume on every rank
    m, u, ci = ph.mapping, ph.u, ph.ci
    del ph
    torch.cuda.empty_cache()
    tau = tau_baseline()
    stream = torch.cuda.current_stream(dev)
    ctx = potts.make_context(dev.index, stream=stream.cuda_stream)
    cuts = native_cuts(m, dist_.world)
    cols, span = native_bounds(m, cuts, dist_.rank)
    comm = nccl_comm(dist_.rank, dist_.world, dev.index) if dist_.world > 1 else None
    opts = {"arith": args.arith, "storage": args.storage, "gap_every": args.gap_every, "prefetch": args.prefetch}
    shard = Shard(ctx, m, cuts, dist_.rank, u.data_ptr() + 4 * span[0], ci, LAMBDA, tau, tau, **opts)
    if comm is not None:
        shard.use_nccl(comm)
    lab = torch.empty(shard.local_span, dtype=torch.uint8, device=dev)
    for _ in range(args.warmup):
        run_shards([shard], args.iters, label_ptrs=[lab.data_ptr()])
    torch.cuda.synchronize(dev)
    dist_.barrier()
    clocks = ClockSampler(dev.index)
    clocks.start()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    stats = [run_shards([shard], args.iters, label_ptrs=[lab.data_ptr()]) for _ in range(args.steps)]
    e1.record(stream)
    torch.cuda.synchronize(dev)
    dist_.barrier()
    clk = clocks.stop()
    t_max = dist_.reduce(e0.elapsed_time(e1) / 1000.0, "max")
    vox = m.data_size
    value = float(vox) * args.iters * args.steps / t_max / 1e9
    own_vox = int(m.base[cols[3]] - m.base[cols[2]]) // m.nstride * m.n_images
    iter_s = sum(s.loop_ms for s in stats) / 1000.0 / max(sum(s.loop_iters for s in stats), 1)
    bpv = bytes_per_voxel_iter("fused", 3, args.storage)
    achieved = dist_.reduce(bpv * own_vox / iter_s / 1e9, "sum")
    peaks = measured_peaks()
    shard.close()
    destroy_comm(comm)
    if dist_.rank == 0:
        out = {"metric": METRIC, "value": round(value, 3), "unit": UNIT, "n_gpus": dist_.world, "steps": args.steps,
               "warmup": args.warmup, "ms_per_step": round(1000 * t_max / args.steps, 2), "higher_is_better": True,
               "scaling": "strong", "vs_baseline": None,
               "dtype": "f32" if args.storage == "f32" else f"f32 math, {args.storage} state", "data": "synthetic",
               "config": {"workload": "potts_k3_768x768x1024_r370_column_shards", "in_mask_voxels": vox,
                          "iters": args.iters, "gap_every": args.gap_every, "arith": args.arith,
                          "storage": args.storage, "parallelism": f"column shards x{dist_.world} (NCCL halos)",
                          "cuts": cuts, "l2": "inputs larger than L2"},
               "roofline": {"bound": "hbm", "achieved": round(achieved, 1),
                            "peak": peaks["hbm_gbs"] * dist_.world, "unit": "GB/s",
                            "frac": round(achieved / (peaks["hbm_gbs"] * dist_.world), 4), "traffic": None,
                            "kernel": "potts::fused_tiled_kernel (per shard)", "bytes_per_voxel_iter": bpv,
                            "avg_iter_ms_rank0": round(iter_s * 1000, 4),
                            "peak_source": f"{peaks['source']} (MEASURED_PEAKS.json hbm_gbs) x ranks"},
               "e2e": None, "gpu_launches": sum(s.total_launches for s in stats), "clocks": clk,
               "cpu_baseline": None,
               "quality": {"final_sqrt_max_dV2": stats[-1].dq_last,
                           "energy_last": stats[-1].energy_trace[-1].tolist()
                           if stats[-1].energy_trace is not None else None}}
        print(json.dumps(out), flush=True)
    ctx.close()
    dist_.close()


def main():
    args = parse_args()
    d = Dist()
    if args.impl == "reference":
        run_reference(args, d)
        return
    if args.shard:
        run_shard(args, d)
        return
    if args.workload == "config3":
        run_batch(args, d)
        return
    if args.workload == "config4":
        run_adjoint(args, d)
        return
    if args.workload in ("tv", "tvmid"):
        run_tv(args, d)
        return
    if args.workload in ("fieldio", "fieldiomid"):
        run_fieldio(args, d)
        return
    if args.workload in ("labels", "labelsmid"):
        run_labels(args, d)
        return
    run_ours(args, d)


if __name__ == "__main__":
    main()
