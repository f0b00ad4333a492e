"""Benchmark of the OMW deconvolution hot path (one JSON line on rank 0).

Workload (default, ``--workload omw_llsm``): one 512x512x256 (x,y,z) uint16 volume, 20 000 Gaussian
puncta over a sinusoid background with Poisson noise, a 64x64x101 two-lobed PSF, OMW RL with 2
iterations, background 100, uint16 output.  A "step" deconvolves one volume.

  value  : Mvoxel/s with the input resident in HBM (device-pointer C-ABI call per step, CUDA events on
           the library's stream, max over ranks).  The working set (0.9 GB) is far larger than L2.
  e2e    : Mvoxel/s through the host-buffer C-ABI (pinned host input and output; H2D of the raw volume
           and D2H of the result of every step inside the timed region): the steps are submitted with
           pk_decon_submit, so step k+1's upload and step k-1's download overlap step k's compute;
           one synchronous pk_decon_lucy_omw call at a time is reported beside it.
  roofline: the dominant kernel's algorithmic HBM bytes per launch / its mean CUDA-event duration.
  cpu_baseline: the CPU restatement of the reference (oracle, float32, scipy.fft on all host cores)
           on one full volume, OTFs cached as the reference caches them.
  cufft_comparator: the same iteration written with torch.fft (cuFFT) + elementwise ops on the same
           resident input, timed the same way; a comparator only.

``--impl reference`` times the reference's CPU path (the oracle restatement; MATLAB is not available)
on the host cores with the same metric.  Under torchrun every rank runs an independent replica
(the path shards by volume; no data-path collective): weak scaling.
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

METRIC = "deconvolved Mvoxel/s (OMW, 2 iter) @rel-L2<=1e-4"
ITERS = 2
BACKGROUND = 100.0


def _peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            p = json.load(f)
        return float(p["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


class ClockSampler:
    """nvidia-smi clocks / throttle reasons sampled during the timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
         "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
         "clocks_event_reasons.sw_power_cap")

    def __init__(self, device):
        self.device = device
        self.rows = []
        self.proc = None
        self.thread = None

    def start(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.device}", f"--query-gpu={self.Q}",
                                          "--format=csv,noheader,nounits", "-lms", "100"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except Exception:
            self.proc = None
            return
        self.thread = threading.Thread(target=self._read, daemon=True)
        self.thread.start()

    def _read(self):
        for line in self.proc.stdout:
            self.rows.append([c.strip() for c in line.split(",")])

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        if self.thread:
            self.thread.join(timeout=2)
        sm, mx, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for r in self.rows:
            try:
                sm.append(float(r[1]))
                mx.append(float(r[2]))
                for n, v in zip(names, r[5:9]):
                    if v.lower().startswith("active"):
                        reasons.add(n)
            except Exception:
                continue
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": sorted(reasons), "samples": len(sm)}


WB = dict(alpha=0.005, beta=1e-3, n=8, res_flag=1)   # Wiener-Butterworth backprojector, Butterworth order 8


def make_workload(seed, reference=False):
    """The headline volume, its PSF and the Wiener-Butterworth backprojector of that PSF (generated
    by the library for our arm, by the CPU restatement for the reference arm)."""
    from petakit5d_b200 import synth
    vol, psf = synth.single_volume_workload("omw_llsm", seed=seed)
    if reference:
        from oracle import backprojector as OB
        pb, _ = OB.wb_backprojector(psf, alpha=WB["alpha"], beta=WB["beta"], n=WB["n"], res_flag=WB["res_flag"])
    else:
        from petakit5d_b200 import backprojector as B
        pb, _ = B.BackProjector(psf, "wiener-butterworth", WB["alpha"], WB["beta"], WB["n"], WB["res_flag"])
    return vol, psf, np.asfortranarray(pb.astype(np.float32))


def cpu_restatement_rate(vol, psf, psf_b, steps=1, warmup=0):
    """Oracle float32 OMW on host cores (OTFs prepared once, as the reference's persistent cache does)."""
    from oracle import decon as O
    shape = vol.shape
    otf_f = O.psf2otf_half(O.normalize_psf(psf, np.float32), shape, np.float32)
    otf_b = O.psf2otf_half(O.normalize_psf(psf_b, np.float32), shape, np.float32)
    eps = np.float32(O.EPS)

    def one():
        I, _ = O.preprocess(vol, BACKGROUND, False, np.float32)
        J = I
        for _ in range(ITERS):
            CX = np.fmax(O.conv_half(J, otf_f), eps)
            J = np.fmax(O.conv_half(I / CX, otf_b) * J, np.float32(0))
        one.J = J
        return O.to_uint16(J)

    for _ in range(warmup):
        one()
    t0 = time.perf_counter()
    for _ in range(steps):
        one()
    dt = (time.perf_counter() - t0) / steps
    cpu_restatement_rate.J = one.J          # the float32 result before the uint16 conversion
    return np.prod(shape) / dt / 1e6, dt


def torch_omw(I16, otf_f, otf_b, iters):
    """cuFFT comparator: the same OMW iteration with torch.fft on a (nz, nx, ny) tensor."""
    import torch
    I = (I16.to(torch.int32) - int(BACKGROUND)).clamp_min(0).to(torch.float32)
    J = I
    shp = I.shape
    for _ in range(iters):
        CX = torch.fft.irfftn(torch.fft.rfftn(J) * otf_f, s=shp).clamp_min(2.0 ** -52)
        J = (torch.fft.irfftn(torch.fft.rfftn(I / CX) * otf_b, s=shp) * J).clamp_min(0)
    return torch.round(J).clamp(0, 65535).to(torch.int32)


def torch_otf(psf, shape_yxz, device):
    """decon_psf2otf at the volume size as a torch half spectrum on the (nz, nx, ny) layout."""
    import torch
    p = np.asarray(psf, np.float64)
    p = (p / p.sum()).astype(np.float32)
    py, px, pz = p.shape
    big = np.zeros(tuple(shape_yxz), np.float32)
    big[:py, :px, :pz] = p
    big = np.roll(big, shift=(-(py // 2), -(px // 2), -(pz // 2)), axis=(0, 1, 2))
    t = torch.from_numpy(np.ascontiguousarray(big.transpose(2, 1, 0))).to(device)
    return torch.fft.rfftn(t)


def run_ours(args, rank, world, device):
    import torch
    from petakit5d_b200 import _lib
    from petakit5d_b200 import decon as D

    vol, psf, psf_b = make_workload(seed=1 + rank)
    ny, nx, nz = vol.shape
    N = ny * nx * nz
    ctx = _lib.Context(device.index)
    stream = torch.cuda.ExternalStream(ctx.stream, device=device)
    d_in = torch.from_numpy(np.ascontiguousarray(vol.T).view(np.int16)).to(device)   # (nz, nx, ny) = column-major
    d_out = torch.empty((nz, nx, ny), dtype=torch.int16, device=device)

    def step():
        D.decon_device("omw", d_in, "uint16", vol.shape, psf, psf_b, ITERS, out=d_out, ctx=ctx,
                       stream=ctx.stream, Background=BACKGROUND)

    torch.cuda.synchronize(device)
    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize(device)

    # -- value: resident input, device-pointer C-ABI call, events on the library stream
    clocks = ClockSampler(device.index)
    clocks.start()
    time.sleep(0.3)
    if world > 1:
        torch.distributed.barrier()
    torch.cuda.synchronize(device)
    l0 = ctx.kernel_launches
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(args.steps):
        step()
    e1.record(stream)
    torch.cuda.synchronize(device)
    launches = ctx.kernel_launches - l0
    if world > 1:
        torch.distributed.barrier()
    # per-pass times: the same K steps again with CUDA events around every kernel (these launch
    # directly, without the call's CUDA graph, so they are timed apart from `value`)
    ctx.profile(True)
    for _ in range(args.steps):
        step()
    torch.cuda.synchronize(device)
    ctx.profile(False)
    clk = clocks.stop()
    ms = e0.elapsed_time(e1) / args.steps
    prof = ctx.profile_read()
    ms_t = torch.tensor([ms], device=device)
    if world > 1:
        torch.distributed.all_reduce(ms_t, op=torch.distributed.ReduceOp.MAX)
    ms = float(ms_t.item())

    # -- e2e: host-buffer C-ABI call, pinned host buffers, copies inside the timed region
    h_in_t = torch.from_numpy(np.ascontiguousarray(vol.T).view(np.int16)).pin_memory()
    h_out_t = torch.empty((nz, nx, ny), dtype=torch.int16).pin_memory()
    h_in = h_in_t.numpy().view(np.uint16).T          # (ny, nx, nz) Fortran view of pinned memory
    h_out = h_out_t.numpy()
    p = D._params({"background": BACKGROUND, "dampfactor": 1.0, "scalefactor": 1.0, "deconoffset": 0.0,
                   "edgeerosion": 0, "save16bit": True, "bbox": None})
    pf = np.asfortranarray(psf, np.float32)
    pb = np.asfortranarray(psf_b, np.float32)

    def e2e_step():
        _lib.check(_lib.lib.pk_decon_lucy_omw(ctx.handle, h_in.ctypes.data, _lib.PK_U16, _lib.i64x3(vol.shape),
                                              pf.ctypes.data, _lib.i64x3(pf.shape), pb.ctypes.data,
                                              _lib.i64x3(pb.shape), ITERS, p, h_out.ctypes.data))

    def submit():
        tk = _lib.C.c_int64()
        _lib.check(_lib.lib.pk_decon_submit(ctx.handle, 1, h_in.ctypes.data, _lib.PK_U16, _lib.i64x3(vol.shape),
                                            pf.ctypes.data, _lib.i64x3(pf.shape), pb.ctypes.data, _lib.i64x3(pb.shape),
                                            ITERS, p, h_out.ctypes.data, _lib.C.byref(tk)))
        return tk.value

    def timed(run):
        if world > 1:
            torch.distributed.barrier()
        torch.cuda.synchronize(device)
        e0.record(stream)
        run()
        e1.record(stream)
        torch.cuda.synchronize(device)
        t = torch.tensor([e0.elapsed_time(e1) / args.steps], device=device)
        if world > 1:
            torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
        return float(t.item())

    # one synchronous call at a time (latency of a single host-buffer call)
    for _ in range(max(1, args.warmup)):
        e2e_step()
    e2e_sync_ms = timed(lambda: [e2e_step() for _ in range(args.steps)])
    h_out[...] = 0

    # e2e: every step submitted through pk_decon_submit; upload of step k+1 and download of step k-1
    # overlap the compute of step k; the stream joins the copy streams before the closing event
    def pipelined():
        tickets = [submit() for _ in range(args.steps)]
        _lib.check(_lib.lib.pk_ctx_join(ctx.handle))
        pipelined.tickets = tickets

    for t in [submit() for _ in range(max(2, args.warmup))]:
        _lib.check(_lib.lib.pk_decon_wait(ctx.handle, t, -1))
    e2e_ms = timed(pipelined)
    for t in pipelined.tickets:
        _lib.check(_lib.lib.pk_decon_wait(ctx.handle, t, -1))
    # the host-buffer result must equal the device-pointer result
    same = bool(np.array_equal(h_out, d_out.cpu().numpy()))

    # the copies alone: the step's H2D and D2H as bare pinned cudaMemcpyAsync on two streams (the
    # floor under `e2e` that no compute overlap can beat)
    d_cp = torch.empty_like(d_in)
    s_up, s_dn = torch.cuda.Stream(device), torch.cuda.Stream(device)
    for _ in range(2):
        with torch.cuda.stream(s_up):
            d_cp.copy_(h_in_t, non_blocking=True)
        with torch.cuda.stream(s_dn):
            h_out_t.copy_(d_out, non_blocking=True)
    torch.cuda.synchronize(device)
    k0, k1, k2 = (torch.cuda.Event(enable_timing=True) for _ in range(3))
    k0.record(s_up)
    s_dn.wait_event(k0)
    for _ in range(args.steps):
        with torch.cuda.stream(s_up):
            d_cp.copy_(h_in_t, non_blocking=True)
        with torch.cuda.stream(s_dn):
            h_out_t.copy_(d_out, non_blocking=True)
    k1.record(s_up)
    k2.record(s_dn)
    torch.cuda.synchronize(device)
    copy_ms = max(k0.elapsed_time(k1), k0.elapsed_time(k2)) / args.steps
    del d_cp

    # one more device call with a float32 output, compared with the oracle after the timed loops
    d_f32 = torch.empty((nz, nx, ny), dtype=torch.float32, device=device)
    D.decon_device("omw", d_in, "uint16", vol.shape, psf, psf_b, ITERS, out=d_f32, ctx=ctx, stream=ctx.stream,
                   Background=BACKGROUND, save16bit=False)
    torch.cuda.synchronize(device)
    J32 = d_f32.cpu().numpy().transpose(2, 1, 0)
    J16 = d_out.cpu().numpy().view(np.uint16).transpose(2, 1, 0)
    del d_f32

    # -- cuFFT comparator on the same resident input
    cst = torch.cuda.Stream(device)
    with torch.cuda.stream(cst):
        of = torch_otf(psf, vol.shape, device)
        ob = torch_otf(psf_b, vol.shape, device)
        I16 = d_in.view(torch.int16).to(torch.int32) & 0xFFFF
        for _ in range(2):
            torch_omw(I16, of, ob, ITERS)
        c0 = torch.cuda.Event(enable_timing=True)
        c1 = torch.cuda.Event(enable_timing=True)
        c0.record(cst)
        for _ in range(args.steps):
            torch_omw(I16, of, ob, ITERS)
        c1.record(cst)
    torch.cuda.synchronize(device)
    cufft_ms = c0.elapsed_time(c1) / args.steps

    peak, peak_kind = _peaks()
    dom = max(prof.items(), key=lambda kv: kv[1]["ms"]) if prof else None
    roof = None
    if dom:
        kind, rec = dom
        per_ms = rec["ms"] / rec["launches"]
        achieved = rec["bytes"] / (per_ms * 1e-3) / 1e9
        traffic = _ncu_traffic().get(kind)
        roof = {"bound": "hbm", "kernel": kind, "achieved": round(achieved, 1), "peak": peak, "unit": "GB/s",
                "frac": round(achieved / peak, 4), "peak_source": peak_kind, "traffic": traffic,
                "algorithmic_bytes_per_launch": rec["bytes"], "ms_per_launch": round(per_ms, 5)}
    call_bytes = N * (64 * ITERS + 12)
    kernels = {k: {"launches": v["launches"], "ms_per_launch": round(v["ms"] / v["launches"], 5),
                   "GBps": round(v["bytes"] / (v["ms"] / v["launches"] * 1e-3) / 1e9, 1),
                   "share": round(v["ms"] / sum(x["ms"] for x in prof.values()), 4)} for k, v in prof.items()}
    return {
        "ms": ms, "N": N, "launches": launches, "clocks": clk, "roofline": roof, "kernels": kernels,
        "autotune": ctx.tune_read(),
        "e2e_ms": e2e_ms, "e2e_sync_ms": e2e_sync_ms, "same": same, "cufft_ms": cufft_ms, "call_bytes": call_bytes, "vol": vol, "psf": psf,
        "psf_b": psf_b, "peak": peak, "peak_kind": peak_kind, "copy_ms": copy_ms, "J32": J32, "J16": J16,
    }


def _ncu_traffic():
    """Per-launch DRAM bytes (read + write) of each pass kind from the committed ncu summary."""
    out = {}
    try:
        with open(os.path.join(ROOT, "profiles", "traffic_omw_llsm_512x512x256.md")) as f:
            for line in f:
                cells = [c.strip() for c in line.strip().strip("|").split("|")]
                if len(cells) == 2 and cells[1].isdigit():
                    out[cells[0]] = int(cells[1])
    except OSError:
        pass
    return out


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-extras", action="store_true",
                    help="leave the batched (96 chunks) and served (Poisson requests) sub-objects off the line")
    ap.add_argument("--workload", default="omw_llsm",
                    choices=["omw_llsm", "rl_small", "batched", "batched_passes", "served", "large", "dsr"])
    ap.add_argument("--rate", type=float, default=200.0, help="served: Poisson arrival rate (requests/s)")
    ap.add_argument("--requests", type=int, default=240, help="served: number of requests")
    ap.add_argument("--ncu-case", action="store_true",
                    help="run two device calls of the workload and exit (the case profiled with ncu)")
    args = ap.parse_args()
    if args.ncu_case:
        import torch
        from petakit5d_b200 import decon as D
        vol, psf, psf_b = make_workload(seed=1)
        d_in = torch.from_numpy(np.ascontiguousarray(vol.T).view(np.int16)).cuda()
        d_out = torch.empty_like(d_in)
        for _ in range(2):
            D.decon_device("omw", d_in, "uint16", vol.shape, psf, psf_b, ITERS, out=d_out, Background=BACKGROUND)
        torch.cuda.synchronize()
        return

    if args.workload != "omw_llsm":
        out = WORKLOADS[args.workload](args)
        if out is not None:
            _emit(out)
        return
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    config = {"workload": "omw_llsm: 512x512x256 (x,y,z) uint16, 20k puncta + sinusoid bg + Poisson, "
                          "64x64x101 lobed PSF, Wiener-Butterworth backprojector (alpha 0.005, beta 1e-3, "
                          "order 8), OMW 2 iterations, uint16 out",
              "volume_xyz": [512, 512, 256], "psf_yxz": [64, 64, 101], "iterations": ITERS,
              "background": BACKGROUND, "parallelism": f"replicas x{world}",
              "l2": "working set 0.9 GB >> 126 MB L2 (no flush needed)"}

    if args.impl == "reference":
        if rank != 0:
            return
        vol, psf, psf_b = make_workload(seed=1, reference=True)
        cores = os.cpu_count()
        rate, dt = cpu_restatement_rate(vol, psf, psf_b, steps=args.steps, warmup=args.warmup)
        print(json.dumps({
            "impl": "reference", "metric": METRIC, "value": round(rate, 3), "unit": "Mvoxel/s",
            "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(dt * 1e3, 1),
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": config,
            "cpu_baseline": {"value": round(rate, 3), "unit": "Mvoxel/s", "cores": cores, "kind": "port",
                             "sample": "one full 512x512x256 volume per step (oracle float32 restatement, "
                                       "scipy.fft on all cores, OTFs cached)"},
            "e2e": {"value": round(rate, 3), "unit": "Mvoxel/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
            "note": "MATLAB (the reference runtime) is not installed; the reference arm is the CPU restatement "
                    "of decon_lucy_omw_function.m (useGPU=false path)",
        }), flush=True)
        return

    import torch
    if world > 1:
        torch.distributed.init_process_group("nccl", init_method="env://", timeout=__import__("datetime").timedelta(seconds=120))
    device = torch.device("cuda", local)
    torch.cuda.set_device(device)
    r = run_ours(args, rank, world, device)
    if world > 1:
        torch.distributed.barrier()
        torch.distributed.destroy_process_group()
    if rank != 0:
        return
    N = r["N"]
    value = N * world / (r["ms"] * 1e-3) / 1e6
    e2e = N * world / (r["e2e_ms"] * 1e-3) / 1e6
    line = {
        "metric": METRIC, "value": round(value, 1), "unit": "Mvoxel/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": round(r["ms"], 4), "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded generator; the reference's demo dataset is "
                                                     "not available offline)",
        "config": config,
        "e2e": {"value": round(e2e, 1), "unit": "Mvoxel/s", "ms_per_step": round(r["e2e_ms"], 4),
                "h2d_bytes_per_step": 2 * N, "d2h_bytes_per_step": 2 * N, "matches_device_call": r["same"],
                "api": "pk_decon_submit per step (pinned host buffers), pk_decon_wait; copies of neighbouring "
                       "steps overlap this step's compute",
                "one_call_at_a_time": {"value": round(N * world / (r["e2e_sync_ms"] * 1e-3) / 1e6, 1),
                                       "ms_per_step": round(r["e2e_sync_ms"], 4), "api": "pk_decon_lucy_omw"}},
        "gpu_launches": r["launches"],
        "roofline": r["roofline"],
        "call_roofline": {"algorithmic_bytes": r["call_bytes"], "achieved": round(r["call_bytes"] / (r["ms"] * 1e-3) / 1e9, 1),
                          "peak": r["peak"], "frac": round(r["call_bytes"] / (r["ms"] * 1e-3) / 1e9 / r["peak"], 4),
                          "unit": "GB/s", "note": "N*(64*iters+12) bytes per call"},
        "kernels": r["kernels"],
        "autotune": r["autotune"],
        "cufft_comparator": {"value": round(N / (r["cufft_ms"] * 1e-3) / 1e6, 1), "unit": "Mvoxel/s",
                             "ms_per_step": round(r["cufft_ms"], 3)},
        "clocks": r["clocks"],
    }
    from oracle import decon as O
    if world == 1 and not args.no_cpu_baseline:
        rate, dt = cpu_restatement_rate(r["vol"], r["psf"], r["psf_b"], steps=1, warmup=0)
        line["cpu_baseline"] = {"value": round(rate, 3), "unit": "Mvoxel/s", "cores": os.cpu_count(), "kind": "port",
                                "sample": "one full 512x512x256 volume (oracle float32, scipy.fft on all cores, "
                                          f"OTFs cached), {dt:.1f} s"}
        ref32 = cpu_restatement_rate.J
    else:
        ref32 = O.decon_lucy_omw(r["vol"], r["psf"], r["psf_b"], ITERS, background=BACKGROUND, save16bit=False,
                                 dtype=np.float32)
    ref64 = O.decon_lucy_omw(r["vol"], r["psf"], np.asarray(r["psf_b"], np.float64), ITERS, background=BACKGROUND,
                             save16bit=False, dtype=np.float64)
    e32, e64 = O.rel_l2(r["J32"], ref32), O.rel_l2(r["J32"], ref64)
    lsb = int(np.max(np.abs(r["J16"].astype(np.int64) - O.to_uint16(ref32).astype(np.int64))))
    line["parity"] = {"rel_l2_vs_fp32_oracle": e32, "rel_l2_vs_fp64_oracle": e64,
                      "fp32_oracle_vs_fp64_oracle": O.rel_l2(ref32, ref64), "uint16_max_lsb_vs_fp32_oracle": lsb,
                      "tolerance": 1e-4, "pass": bool(e32 <= 1e-4 and lsb <= 1),
                      "checked": "a float32-output device call on rank 0's volume after the timed loops, and the "
                                 "timed calls' uint16 output, against the oracle restatement of "
                                 "decon_lucy_omw_function.m:105-113 with the same backprojector"}
    if world == 1 and not args.no_extras:
        # the batched and served patterns of the same library, on their own workloads (compact)
        for name, fn, keys in (("batched", wl_batched, ("value", "unit", "plain_per_chunk", "speedup_vs_plain",
                                                         "batched_equals_plain", "ms_batched", "ms_plain",
                                                         "device_resident", "workload")),
                               ("served", wl_served, ("value", "unit", "latency_ms", "plain_sequential",
                                                      "speedup_vs_plain", "wall_s", "saturated", "device_loop",
                                                      "workload"))):
            try:
                sub = fn(args)
                line[name] = {k: sub[k] for k in keys if k in sub}
            except Exception as e:   # reported, not fatal: the headline line still prints
                line[name] = {"error": repr(e)[:300]}
    line["e2e"]["copy_floor"] = {
        "ms_per_step": round(r["copy_ms"], 4), "value": round(N * world / (r["copy_ms"] * 1e-3) / 1e6, 1),
        "GBps_each_way": round(2 * N / (r["copy_ms"] * 1e-3) / 1e9, 1),
        "note": "the step's H2D and D2H alone: bare pinned copies on two streams, no compute"}
    print(json.dumps(line), flush=True)



# ====================================================================== further workloads
def _events(stream):
    import torch
    return torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)


def _emit(line):
    print(json.dumps(line), flush=True)


_T0 = time.perf_counter()


def _log(msg):
    print(f"[{time.perf_counter() - _T0:8.1f}s] {msg}", file=sys.stderr, flush=True)


def _u16_dev(vol, device):
    import torch
    return torch.from_numpy(np.ascontiguousarray(vol.T).view(np.int16)).to(device)


def wl_rl_small(args):
    """Config 1: one 128x128x64 volume, 31x31x41 Gaussian PSF, Biggs RL 20 iterations, float32 out."""
    import torch
    from petakit5d_b200 import _lib
    from petakit5d_b200 import decon as D
    from petakit5d_b200 import synth
    from oracle import decon as O
    if args.impl == "reference":
        vol, psf = synth.single_volume_workload("rl_small", seed=1)
        t0 = time.perf_counter()
        for _ in range(max(1, args.steps)):
            O.decon_lucy(vol, psf, 20, background=100, save16bit=False)
        dt = (time.perf_counter() - t0) / max(1, args.steps)
        v = vol.size / dt / 1e6
        _emit({"impl": "reference", "metric": "deconvolved Mvoxel/s (RL, 20 iter)", "value": round(v, 3),
               "unit": "Mvoxel/s", "workload": "rl_small", "cpu_baseline": {"value": round(v, 3), "unit": "Mvoxel/s",
               "cores": os.cpu_count(), "kind": "port", "sample": "one 128x128x64 volume per step"}})
        return
    device = torch.device("cuda", 0)
    vol, psf = synth.single_volume_workload("rl_small", seed=1)
    ctx = _lib.Context(0)
    stream = torch.cuda.ExternalStream(ctx.stream, device=device)
    d_in = _u16_dev(vol, device)
    d_out = torch.empty(vol.T.shape, dtype=torch.float32, device=device)
    step = lambda: D.decon_device("rl", d_in, "uint16", vol.shape, psf, None, 20, out=d_out, ctx=ctx,
                                  stream=ctx.stream, Background=100.0, save16bit=False)
    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize()
    e0, e1 = _events(stream)
    e0.record(stream)
    for _ in range(args.steps):
        step()
    e1.record(stream)
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1) / args.steps
    J = d_out.cpu().numpy().transpose(2, 1, 0)
    ref = O.decon_lucy(vol, psf, 20, background=100, save16bit=False, dtype=np.float32)
    ref64 = O.decon_lucy(vol, psf, 20, background=100, save16bit=False, dtype=np.float64)
    t0 = time.perf_counter()
    O.decon_lucy(vol, psf, 20, background=100, save16bit=False)
    cpu_dt = time.perf_counter() - t0
    _emit({"metric": "deconvolved Mvoxel/s (RL, 20 iter)", "workload": "rl_small 128x128x64, 31x31x41 PSF",
           "value": round(vol.size / (ms * 1e-3) / 1e6, 1), "unit": "Mvoxel/s", "ms_per_step": round(ms, 4),
           "rel_l2_vs_fp32_oracle": O.rel_l2(J, ref), "rel_l2_vs_fp64_oracle": O.rel_l2(J, ref64),
           "cpu_baseline": {"value": round(vol.size / cpu_dt / 1e6, 3), "unit": "Mvoxel/s", "cores": os.cpu_count(),
                            "kind": "port", "sample": "one volume"}})


def _chunk_set(device, n_chunks=96, seed=3, border=16):
    """Config 3 chunks generated on the GPU, copied to pinned host memory (numpy views)."""
    import torch
    from petakit5d_b200 import synth
    rng = np.random.Generator(np.random.PCG64(seed))
    psfs = [synth.gaussian_psf((31, 31, 41), s, 3.0) for s in (1.3, 1.5, 1.8)]
    chunks, ids, boxes, pinned = [], [], [], []
    density = 200.0 / (128 * 128 * 64)
    for i in range(n_chunks):
        cy, cx = int(rng.choice((192, 256, 320, 384))), int(rng.choice((192, 256, 320, 384)))
        cz = int(rng.choice((96, 128, 192, 256)))
        pid = int(rng.integers(0, 3))
        shape = (cy + 2 * border, cx + 2 * border, cz + 2 * border)
        t = synth.puncta_volume_torch(shape, int(round(density * np.prod(shape))), psfs[pid], seed * 1000 + i,
                                      100.0, device=device)
        h = t.cpu().pin_memory()
        pinned.append(h)
        chunks.append(h.numpy().view(np.uint16).T)      # (ny, nx, nz) Fortran view of pinned memory
        ids.append(pid)
        boxes.append([border + 1, border + 1, border + 1, border + cy, border + cx, border + cz])
    torch.cuda.empty_cache()
    return chunks, pinned, psfs, ids, boxes


def wl_batched(args):
    """Config 3: 96 uneven chunks with 16-voxel borders, 3 PSFs, OMW 2 iterations; batched call
    (shared launches, pipelined copies) against 96 plain per-chunk calls, host buffers both ways."""
    import torch
    from petakit5d_b200 import _lib
    from petakit5d_b200 import backprojector as B
    from petakit5d_b200 import chunking as K
    from petakit5d_b200 import decon as D
    device = torch.device("cuda", 0)
    _log("batched: generating 96 chunks")
    chunks, pinned, psfs, ids, boxes = _chunk_set(device)
    _log("batched: generated")
    if args.impl == "reference":
        from oracle import backprojector as OB
        from oracle import decon as O
        bps = [OB.omw_backprojector_generation(p, 0.005, False, otf_cum_thresh=0.6)[0] for p in psfs]
        t0 = time.perf_counter()
        nvox = 0
        sample = chunks[:4]
        for c, pid, bb in zip(sample, ids[:4], boxes[:4]):
            O.decon_lucy_omw(c, psfs[pid], bps[pid], 2, background=100, bbox=bb)
            nvox += (bb[3] - bb[0] + 1) * (bb[4] - bb[1] + 1) * (bb[5] - bb[2] + 1)
        v = nvox / (time.perf_counter() - t0) / 1e6
        _emit({"impl": "reference", "metric": "batched OMW Mvoxel/s (output core voxels)", "value": round(v, 3),
               "unit": "Mvoxel/s", "workload": "batched", "cpu_baseline": {"value": round(v, 3), "unit": "Mvoxel/s",
               "cores": os.cpu_count(), "kind": "port", "sample": "first 4 of the 96 chunks"}})
        return
    bps = [B.omw_backprojector_generation(p, 0.005, False, OTFCumThresh=0.6)[0] for p in psfs]
    ctx = _lib.Context(0)
    stream = torch.cuda.ExternalStream(ctx.stream, device=device)
    core = sum((b[3] - b[0] + 1) * (b[4] - b[1] + 1) * (b[5] - b[2] + 1) for b in boxes)
    outs = [np.empty((b[3] - b[0] + 1, b[4] - b[1] + 1, b[5] - b[2] + 1), np.uint16, order="F") for b in boxes]
    pouts = []
    for i, o in enumerate(outs):       # pinned outputs
        t = torch.empty(o.shape[::-1], dtype=torch.int16).pin_memory()
        pouts.append(t)
        outs[i] = t.numpy().view(np.uint16).T

    def batched():
        K.batch_decon(chunks, psfs, ids, 2, "omw", bps, boxes, ctx=ctx, outputs=outs, Background=100)

    def plain():
        for c, pid, bb, o in zip(chunks, ids, boxes, outs):
            p = D._params({"background": 100.0, "dampfactor": 1.0, "scalefactor": 1.0, "deconoffset": 0.0,
                           "edgeerosion": 0, "save16bit": True, "bbox": bb})
            pf = np.asfortranarray(psfs[pid], np.float32)
            pb = np.asfortranarray(bps[pid], np.float32)
            _lib.check(_lib.lib.pk_decon_lucy_omw(ctx.handle, c.ctypes.data, _lib.PK_U16, _lib.i64x3(c.shape),
                                                  pf.ctypes.data, _lib.i64x3(pf.shape), pb.ctypes.data,
                                                  _lib.i64x3(pb.shape), 2, p, o.ctypes.data))

    # the same batch with every chunk and output resident on the device (no copies): the compute bound
    d_chunks = [pc.to(device) for pc in pinned]
    d_outs = [torch.empty(o.shape[::-1], dtype=torch.int16, device=device) for o in outs]
    arr = (_lib.Chunk * len(chunks))()
    for i, (c, bb) in enumerate(zip(chunks, boxes)):
        arr[i].in_ = d_chunks[i].data_ptr()
        arr[i].dims = _lib.i64x3(c.shape)
        arr[i].psf_id = int(ids[i])
        arr[i].has_bbox = 1
        for k in range(6):
            arr[i].bbox[k] = int(bb[k])
        arr[i].out = d_outs[i].data_ptr()
    pfs = [np.asfortranarray(q, np.float32) for q in psfs]
    pbs = [np.asfortranarray(q, np.float32) for q in bps]
    fptrs = (_lib.C.c_void_p * len(pfs))(*[a.ctypes.data for a in pfs])
    bptrs = (_lib.C.c_void_p * len(pbs))(*[a.ctypes.data for a in pbs])
    pdims = np.array([list(a.shape) for a in pfs], dtype=np.int64).ravel()
    pdev = D._params({"background": 100.0, "dampfactor": 1.0, "scalefactor": 1.0, "deconoffset": 0.0,
                      "edgeerosion": 0, "save16bit": True, "bbox": None})

    def resident():
        _lib.check(_lib.lib.pk_batch_decon(ctx.handle, 1, len(chunks), arr, _lib.PK_U16, len(pfs), fptrs, bptrs,
                                           pdims.ctypes.data, 2, pdev, 0, 1))

    res = {}
    for name, fn in (("plain", plain), ("batched", batched), ("resident", resident)):
        fn()                                   # warm-up: OTFs cached
        fn()                                   # second warm-up: repeated programs become graphs
        torch.cuda.synchronize()
        reps = max(1, min(args.steps, 3))
        e0, e1 = _events(stream)
        e0.record(stream)
        for _ in range(reps):
            fn()
        e1.record(stream)
        torch.cuda.synchronize()
        res[name] = e0.elapsed_time(e1) / reps
        _log(f"batched: {name} {res[name]:.1f} ms")
    ref_out = [o.copy() for o in outs]
    batched()
    same = all(np.array_equal(a, b) for a, b in zip(ref_out, outs))
    return ({"metric": "batched OMW Mvoxel/s (output core voxels, host buffers, copies included)",
           "workload": "96 uneven chunks (core x,y in {192..384}, z in {96..256}, +16 borders), 3 PSFs, OMW x2",
           "value": round(core / (res["batched"] * 1e-3) / 1e6, 1), "unit": "Mvoxel/s",
           "plain_per_chunk": round(core / (res["plain"] * 1e-3) / 1e6, 1),
           "speedup_vs_plain": round(res["plain"] / res["batched"], 3), "ms_batched": round(res["batched"], 2),
           "ms_plain": round(res["plain"], 2), "batched_equals_plain": same, "core_voxels": int(core),
           "device_resident": {"value": round(core / (res["resident"] * 1e-3) / 1e6, 1), "unit": "Mvoxel/s",
                               "ms": round(res["resident"], 2),
                               "note": "same batch with chunks and outputs already in HBM (compute bound)"}})


def wl_batched_passes(args):
    """Config 3's batch, chunks and outputs resident in HBM, with every x / z kernel candidate forced
    in turn (PK_TMA_VARIANT; "tuned" = the autotuner's choices): per-pass kernel time by transform
    length and kernel family, one profiled call after two warm-ups per candidate."""
    import torch
    from petakit5d_b200 import _lib
    from petakit5d_b200 import backprojector as B
    from petakit5d_b200 import decon as D
    if args.impl == "reference":
        _emit({"impl": "reference", "unavailable": "per-pass kernel profile of the GPU path (no CPU counterpart)"})
        return None
    os.environ["PK_PROF_DETAIL"] = "1"
    device = torch.device("cuda", 0)
    chunks, pinned, psfs, ids, boxes = _chunk_set(device)
    bps = [B.omw_backprojector_generation(p, 0.005, False, OTFCumThresh=0.6)[0] for p in psfs]
    d_chunks = [pc.to(device) for pc in pinned]
    d_outs = [torch.empty(((b[5] - b[2] + 1), (b[4] - b[1] + 1), (b[3] - b[0] + 1)), dtype=torch.int16, device=device)
              for b in boxes]
    arr = (_lib.Chunk * len(chunks))()
    for i, (c, bb) in enumerate(zip(chunks, boxes)):
        arr[i].in_ = d_chunks[i].data_ptr()
        arr[i].dims = _lib.i64x3(c.shape)
        arr[i].psf_id = int(ids[i])
        arr[i].has_bbox = 1
        for k in range(6):
            arr[i].bbox[k] = int(bb[k])
        arr[i].out = d_outs[i].data_ptr()
    pfs = [np.asfortranarray(q, np.float32) for q in psfs]
    pbs = [np.asfortranarray(q, np.float32) for q in bps]
    fptrs = (_lib.C.c_void_p * 3)(*[a.ctypes.data for a in pfs])
    bptrs = (_lib.C.c_void_p * 3)(*[a.ctypes.data for a in pbs])
    pdims = np.array([list(a.shape) for a in pfs], dtype=np.int64).ravel()
    p = D._params({"background": 100.0, "dampfactor": 1.0, "scalefactor": 1.0, "deconoffset": 0.0,
                   "edgeerosion": 0, "save16bit": True, "bbox": None})
    res = {}
    for v in ("tuned", "-1", "0", "1", "2"):
        if v == "tuned":
            os.environ.pop("PK_TMA_VARIANT", None)
        else:
            os.environ["PK_TMA_VARIANT"] = v
        ctx = _lib.Context(0)

        def run():
            _lib.check(_lib.lib.pk_batch_decon(ctx.handle, 1, len(chunks), arr, _lib.PK_U16, 3, fptrs, bptrs,
                                               pdims.ctypes.data, 2, p, 0, 1))

        run()
        run()
        torch.cuda.synchronize()
        ctx.profile(True)
        run()
        torch.cuda.synchronize()
        ctx.profile(False)
        prof = ctx.profile_read()
        res[v] = {"total_ms": round(sum(x["ms"] for x in prof.values()), 3),
                  "passes": {k: round(x["ms"], 3) for k, x in sorted(prof.items())}}
        if v == "tuned":
            res[v]["autotune"] = ctx.tune_read()
        del ctx
    os.environ.pop("PK_TMA_VARIANT", None)
    return {"metric": "batched per-pass kernel ms by forced x / z candidate", "workload": "batched_passes",
            "unit": "ms", "candidates": res,
            "note": "kinds are pass@transform-length:family (tma, rio = register-IO, rolled / yreg y kernels, "
                    "-1k = 1024-point tiles); -1 = register-IO forced, 0-2 = TMA variant where the plan has it"}


def wl_served(args):
    """Config 4: open-loop Poisson requests (90% chunk sizes, 10% 768x768x384; 80% OMW x2, 20% RL x10;
    3 PSFs; 150 GB budget) through the continuous-batching server, against the same requests run one
    after another with the plain host call."""
    import threading
    import torch
    from petakit5d_b200 import _lib
    from petakit5d_b200 import backprojector as B
    from petakit5d_b200 import serve as SV
    from petakit5d_b200 import synth
    device = torch.device("cuda", 0)
    rng = np.random.Generator(np.random.PCG64(17))
    psfs = [synth.gaussian_psf((31, 31, 41), s, 3.0) for s in (1.3, 1.5, 1.8)]
    bps = [B.omw_backprojector_generation(p, 0.005, False, OTFCumThresh=0.6)[0] for p in psfs]
    pool = {}
    keep = []

    def volume(shape):
        if shape not in pool:
            t = synth.puncta_volume_torch(shape, int(np.prod(shape) * 200 / (128 * 128 * 64)), psfs[0],
                                          len(pool) + 5, 100.0, device=device)
            h = t.cpu().pin_memory()
            keep.append(h)
            pool[shape] = h.numpy().view(np.uint16).T
        return pool[shape]

    reqs = []
    for i in range(args.requests):
        if rng.random() < 0.9:
            shape = (int(rng.choice((192, 256, 320, 384))) + 32, int(rng.choice((192, 256, 320, 384))) + 32,
                     int(rng.choice((96, 128, 192, 256))) + 32)
        else:
            shape = (768, 768, 384)
        method = "omw" if rng.random() < 0.8 else "rl"
        reqs.append((volume(shape), int(rng.integers(0, 3)), method, 2 if method == "omw" else 10))
    torch.cuda.empty_cache()
    arrivals = np.cumsum(rng.exponential(1.0 / args.rate, size=len(reqs)))
    nvox = sum(int(np.prod(r[0].shape)) for r in reqs)
    ctx = _lib.Context(0)
    srv = SV.Server(ctx, budget_bytes=150e9, max_batch=64, borrow_inputs=True)
    for i in range(3):
        srv.add_psf(i, psfs[i], bps[i])
    _log(f"served: {len(reqs)} requests, {len(pool)} distinct sizes generated")
    # warm-up: every (size, PSF, method) combination once, so the OTFs are cached as a running
    # server's would be, and the kernels are loaded
    seen = {}
    for v, pid, m, _ in reqs:
        seen[(v.shape, pid, m)] = v
    warm = [srv.submit(v, pid, m, 1, Background=100) for (shp, pid, m), v in seen.items()]
    for w in warm:
        srv.wait(w)
    _log(f"served: warm-up of {len(warm)} combinations done")
    outs = {}
    for v, _, _, _ in reqs:
        if v.shape not in outs:
            t = torch.empty(v.shape[::-1], dtype=torch.int16).pin_memory()
            keep.append(t)
            outs[v.shape] = t.numpy().view(np.uint16).T
    import queue

    def phase(arr, srv):
        """Submit request i at arrival time arr[i] (seconds from the start); returns (wall s, latencies)."""
        lat = [None] * len(reqs)
        ids = [None] * len(reqs)
        done = threading.Semaphore(0)
        q = queue.Queue()

        def waiter():
            while True:
                i = q.get()
                if i is None:
                    return
                _, ms = srv.wait(ids[i], out=outs[reqs[i][0].shape])
                lat[i] = ms
                done.release()

        ws = [threading.Thread(target=waiter, daemon=True) for _ in range(8)]
        for w in ws:
            w.start()
        t0 = time.perf_counter()
        for i, (v, pid, m, it) in enumerate(reqs):
            now = time.perf_counter() - t0
            if arr[i] > now:
                time.sleep(arr[i] - now)
            ids[i] = srv.submit(v, pid, m, it, Background=100)
            q.put(i)
        for _ in reqs:
            done.acquire()
        wall = time.perf_counter() - t0
        for _ in ws:
            q.put(None)
        return wall, lat

    # the same requests, one plain host call after another (each (size, PSF, method) warmed up first,
    # as the server's were: OTFs cached, kernels loaded, variants tuned)
    def plain_call(v, pid, m, it):
        o = outs[v.shape]
        p = D_params()
        pf = np.asfortranarray(psfs[pid], np.float32)
        if m == "omw":
            pb = np.asfortranarray(bps[pid], np.float32)
            _lib.check(_lib.lib.pk_decon_lucy_omw(ctx.handle, v.ctypes.data, _lib.PK_U16, _lib.i64x3(v.shape),
                                                  pf.ctypes.data, _lib.i64x3(pf.shape), pb.ctypes.data,
                                                  _lib.i64x3(pb.shape), it, p, o.ctypes.data))
        else:
            _lib.check(_lib.lib.pk_decon_lucy(ctx.handle, v.ctypes.data, _lib.PK_U16, _lib.i64x3(v.shape),
                                              pf.ctypes.data, _lib.i64x3(pf.shape), it, p, o.ctypes.data, None))

    def plain_all():
        t1 = time.perf_counter()
        for v, pid, m, it in reqs:
            plain_call(v, pid, m, it)
        return time.perf_counter() - t1

    for (shp, pid, m), v in seen.items():
        plain_call(v, pid, m, 1)
    plain = plain_all()
    _log(f"served: the plain calls one after another took {plain:.2f} s")
    # warm-up of the multi-volume rounds: the whole request set once, untimed, so the autotuner's
    # choices for rounds of many volumes are made here and not inside the timed phases
    phase(np.zeros(len(reqs)), srv)
    timed0 = sum(1 for r in ctx.tune_read() if r.get("source") == "timed")
    wall, lat = phase(arrivals, srv)
    _log(f"served: {len(reqs)} requests done in {wall:.2f} s")
    # the same requests all at once: the server's throughput when arrivals do not limit it
    wall_sat, lat_sat = phase(np.zeros(len(reqs)), srv)
    _log(f"served: {len(reqs)} requests submitted at once done in {wall_sat:.2f} s")
    tuned_in_phases = sum(1 for r in ctx.tune_read() if r.get("source") == "timed") - timed0
    st = srv.stats()
    srv.close()
    # the same two phases through the device-resident request loop (a dispatcher kernel launches
    # each admitted request's pass graph from the device)
    dsrv = SV.Server(ctx, budget_bytes=150e9, max_batch=64, borrow_inputs=True, device_loop=True)
    for i in range(3):
        dsrv.add_psf(i, psfs[i], bps[i])
    for w in [dsrv.submit(v, pid, m, 1, Background=100) for (shp, pid, m), v in seen.items()]:
        dsrv.wait(w)
    dwall, dlat = phase(arrivals, dsrv)
    dwall_sat, dlat_sat = phase(np.zeros(len(reqs)), dsrv)
    dloop = dsrv.loop_status()
    dsrv.close()
    _log(f"served (device loop): {dwall:.2f} s open loop, {dwall_sat:.2f} s all at once")
    plain_after = plain_all()
    _log(f"served: the plain calls again after serving took {plain_after:.2f} s")
    L = np.array(lat)
    return ({"metric": "served Mvoxel/s and request latency", "workload":
           f"{len(reqs)} open-loop Poisson requests at {args.rate} req/s (90% chunk sizes, 10% 768x768x384; 80% OMW x2, "
           "20% RL x10; 3 PSFs; 150 GB budget)",
           "value": round(nvox / wall / 1e6, 1), "unit": "Mvoxel/s",
           "latency_ms": {"p50": round(float(np.percentile(L, 50)), 2), "p95": round(float(np.percentile(L, 95)), 2),
                          "p99": round(float(np.percentile(L, 99)), 2), "max": round(float(L.max()), 2)},
           "plain_sequential": round(nvox / plain / 1e6, 1), "speedup_vs_plain": round(plain / wall, 3),
           "wall_s": round(wall, 3), "plain_s": round(plain, 3), "rounds": st["rounds"],
           "peak_inflight_GB": round(st["peak_inflight_bytes"] / 1e9, 2), "plain_s_after_serving": round(plain_after, 3),
           "autotune_timings_while_serving": tuned_in_phases,
           "saturated": {"value": round(nvox / wall_sat / 1e6, 1), "unit": "Mvoxel/s",
                         "speedup_vs_plain": round(plain / wall_sat, 3), "wall_s": round(wall_sat, 3),
                         "latency_ms": {"p50": round(float(np.percentile(lat_sat, 50)), 2),
                                        "p99": round(float(np.percentile(lat_sat, 99)), 2)},
                         "note": "the same requests submitted at once (throughput not limited by arrivals)"},
           "device_loop": {"value": round(nvox / dwall / 1e6, 1), "unit": "Mvoxel/s",
                           "speedup_vs_plain": round(plain / dwall, 3), "wall_s": round(dwall, 3),
                           "latency_ms": {"p50": round(float(np.percentile(dlat, 50)), 2),
                                          "p95": round(float(np.percentile(dlat, 95)), 2),
                                          "p99": round(float(np.percentile(dlat, 99)), 2)},
                           "saturated": {"value": round(nvox / dwall_sat / 1e6, 1),
                                         "speedup_vs_plain": round(plain / dwall_sat, 3)},
                           "dispatcher_instances": dloop["instances"],
                           "note": "the same requests through the device-resident loop: a dispatcher kernel "
                                   "launches each admitted request's pass graph from the device"}})


DSR = dict(angle=32.45, dz=0.3, xy=0.108, reverse=True)   # the reference demo's deskew / rotate settings


def wl_dsr(args):
    """Deskew / rotate of the headline volume's deconvolution (deskewRotateFrame3D, the demo's light-
    sheet geometry: 32.45 deg, dz 0.3 um, 0.108 um pixels, reverse; |dx| = 2.34 px > 2, so slices are
    interpolated in the skewed space first), uint16 in and out, everything resident on the device.
    The rate is output voxels per second; each kernel's algorithmic bytes read the input (and the
    interpolated slices) once and write each output once."""
    import torch
    from petakit5d_b200 import _lib
    from petakit5d_b200 import decon as D
    from petakit5d_b200 import deskew as G
    from oracle import deskew as OD
    if args.impl == "reference":
        vol, _, _ = make_workload(seed=1, reference=True)
        sub = np.asfortranarray(vol[:, :, :24])
        t0 = time.perf_counter()
        out = OD.deskew_rotate_frame3d(sub, DSR["angle"], DSR["dz"], DSR["xy"], reverse=DSR["reverse"], save16bit=True)
        v = out.size / (time.perf_counter() - t0) / 1e6
        _emit({"impl": "reference", "metric": "deskew/rotate output Mvoxel/s", "value": round(v, 3), "unit": "Mvoxel/s",
               "workload": "dsr", "cpu_baseline": {"value": round(v, 3), "unit": "Mvoxel/s", "cores": 1, "kind": "port",
                                                   "sample": "the first 24 z slices of the volume"}})
        return
    device = torch.device("cuda", 0)
    vol, psf, psf_b = make_workload(seed=1)
    ctx = _lib.Context(0)
    stream = torch.cuda.ExternalStream(ctx.stream, device=device)
    d_in = _u16_dev(vol, device)
    d_j = torch.empty_like(d_in)
    D.decon_device("omw", d_in, "uint16", vol.shape, psf, psf_b, ITERS, out=d_j, ctx=ctx, stream=ctx.stream,
                   Background=BACKGROUND)
    kw = dict(reverse=DSR["reverse"], save16bit=True, ctx=ctx, stream=ctx.stream)
    dims = G.deskew_rotate_device(d_j, "uint16", vol.shape, DSR["angle"], DSR["dz"], DSR["xy"], **kw)
    d_o = torch.empty(int(np.prod(dims)), dtype=torch.int16, device=device)
    step = lambda: G.deskew_rotate_device(d_j, "uint16", vol.shape, DSR["angle"], DSR["dz"], DSR["xy"], d_out=d_o, **kw)
    for _ in range(max(3, args.warmup)):
        step()
    torch.cuda.synchronize()
    e0, e1 = _events(stream)
    steps = max(1, args.steps)
    e0.record(stream)
    for _ in range(steps):
        step()
    e1.record(stream)
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1) / steps
    ctx.profile(True)
    step()
    torch.cuda.synchronize()
    prof = ctx.profile_read()
    ctx.profile(False)
    p = OD.plan(vol.shape, DSR["angle"], DSR["dz"], DSR["xy"], reverse=DSR["reverse"])
    _, _, nint = OD.interp_indexing(p["nz_total"], p["stepsize"])
    n_out = int(np.prod(dims))
    peak = _peaks()[0]
    kern = {}
    for k, v in (prof or {}).items():
        gbs = v["bytes"] / (v["ms"] * 1e-3) / 1e9
        kern[k] = {"ms": round(v["ms"], 4), "algorithmic_MB": round(v["bytes"] / 1e6, 1), "GB/s": round(gbs, 1),
                   "frac_of_measured_hbm": round(gbs / peak, 3)}
    # CPU sample for scale: the oracle on the first 24 z slices
    sub = np.asfortranarray(d_j.cpu().numpy().view(np.uint16).T[:, :, :24])
    t0 = time.perf_counter()
    osub = OD.deskew_rotate_frame3d(sub, DSR["angle"], DSR["dz"], DSR["xy"], reverse=DSR["reverse"], save16bit=True)
    cpu = osub.size / (time.perf_counter() - t0) / 1e6
    _emit({"metric": "deskew/rotate output Mvoxel/s", "workload": "dsr: OMW x2 result of the 512x512x256 volume, "
           "angle 32.45, dz 0.3, 0.108 um, reverse, uint16 in/out, skewed-space interpolation (step 1/2)",
           "value": round(n_out / (ms * 1e-3) / 1e6, 1), "unit": "Mvoxel/s", "ms_per_step": round(ms, 4),
           "out_dims": list(dims), "interpolated_slices": nint, "kernels": kern,
           "cpu_baseline": {"value": round(cpu, 3), "unit": "Mvoxel/s", "cores": 1, "kind": "port",
                            "sample": "the first 24 z slices of the deconvolved volume"}})


def D_params():
    from petakit5d_b200 import decon as D
    return D._params({"background": 100.0, "dampfactor": 1.0, "scalefactor": 1.0, "deconoffset": 0.0,
                      "edgeerosion": 0, "save16bit": True, "bbox": None})


def wl_large(args):
    """Config 5: 2048x2048x1024 volume (2M puncta), OMW x2 with the small PSF, whole volume resident
    in HBM and as 512^3 chunks with 32-voxel overlap through the batched path (device buffers)."""
    import torch
    from petakit5d_b200 import _lib
    from petakit5d_b200 import backprojector as B
    from petakit5d_b200 import chunking as K
    from petakit5d_b200 import decon as D
    from petakit5d_b200 import synth
    device = torch.device("cuda", 0)
    shape = (2048, 2048, 1024)
    psf = synth.gaussian_psf((31, 31, 41), 1.3, 3.0)
    bp = B.omw_backprojector_generation(psf, 0.005, False, OTFCumThresh=0.6)[0]
    _log("large: generating 2048x2048x1024")
    d_in = synth.puncta_volume_torch(shape, 2_000_000, psf, 7, 100.0, device=device, gaussian_psf_sigmas=(1.3, 3.0))
    torch.cuda.empty_cache()
    _log("large: generated")
    N = int(np.prod(shape))
    ctx = _lib.Context(0)
    stream = torch.cuda.ExternalStream(ctx.stream, device=device)
    d_out = torch.empty_like(d_in)
    run = lambda: D.decon_device("omw", d_in, "uint16", shape, psf, bp, 2, out=d_out, ctx=ctx, stream=ctx.stream,
                                 Background=100.0)
    run()
    torch.cuda.synchronize()
    e0, e1 = _events(stream)
    e0.record(stream)
    run()
    e1.record(stream)
    torch.cuda.synchronize()
    whole_ms = e0.elapsed_time(e1)
    _log(f"large: whole volume {whole_ms:.1f} ms")
    ctx.reset()
    # chunked: 512^3 regions, border 32, through the batched path on device buffers
    bb, rb, _ = K.zarr_chunk_coordinates(shape, (512, 512, 512), (512, 512, 512), None, False, 32)
    chunks, outs, boxes = [], [], []
    for b, r in zip(bb, rb):
        c = d_in[b[2] - 1:b[5], b[1] - 1:b[4], b[0] - 1:b[3]].contiguous()
        chunks.append(c)
        st_ = r[:3] - b[:3] + 1
        en = r[3:] - b[:3] + 1
        boxes.append([*st_, *en])
        outs.append(torch.empty((en[2] - st_[2] + 1, en[1] - st_[1] + 1, en[0] - st_[0] + 1), dtype=torch.int16,
                                device=device))
    n = len(chunks)
    arr = (_lib.Chunk * n)()
    for i, (c, o, bx) in enumerate(zip(chunks, outs, boxes)):
        arr[i].in_ = c.data_ptr()
        arr[i].dims = _lib.i64x3((c.shape[2], c.shape[1], c.shape[0]))
        arr[i].psf_id = 0
        arr[i].has_bbox = 1
        for k in range(6):
            arr[i].bbox[k] = int(bx[k])
        arr[i].out = o.data_ptr()
    pf = np.asfortranarray(psf, np.float32)
    pb = np.asfortranarray(bp, np.float32)
    fp = (_lib.C.c_void_p * 1)(pf.ctypes.data)
    bpp = (_lib.C.c_void_p * 1)(pb.ctypes.data)
    dims = np.array(pf.shape, np.int64)
    p = D_params()
    call = lambda: _lib.check(_lib.lib.pk_batch_decon(ctx.handle, 1, n, arr, _lib.PK_U16, 1, fp, bpp, dims.ctypes.data, 2,
                                                      p, 0, 1))
    call()
    torch.cuda.synchronize()
    e0.record(stream)
    call()
    e1.record(stream)
    torch.cuda.synchronize()
    chunk_ms = e0.elapsed_time(e1)
    _log(f"large: {n} chunks {chunk_ms:.1f} ms")
    stitched = torch.empty_like(d_in)
    for r, o in zip(rb, outs):
        stitched[r[2] - 1:r[5], r[1] - 1:r[4], r[0] - 1:r[3]] = o
    num = den = 0.0
    for z0 in range(0, shape[2], 64):                      # slab-wise: every tensor < 2^31 elements
        a = d_out[z0:z0 + 64].to(torch.int32) & 0xFFFF
        b2 = stitched[z0:z0 + 64].to(torch.int32) & 0xFFFF
        num += float(((a - b2).double() ** 2).sum())
        den += float((a.double() ** 2).sum())
    gap = (num / den) ** 0.5
    # the same gap away from the volume's own faces (a 64-voxel band), where the whole volume's
    # circular transform joins opposite faces and the edge chunks do not
    m = 64
    num = den = 0.0
    for z0 in range(m, shape[2] - m, 64):
        z1 = min(z0 + 64, shape[2] - m)
        a = d_out[z0:z1, m:-m, m:-m].to(torch.int32) & 0xFFFF
        b2 = stitched[z0:z1, m:-m, m:-m].to(torch.int32) & 0xFFFF
        num += float(((a - b2).double() ** 2).sum())
        den += float((a.double() ** 2).sum())
    gap_in = (num / den) ** 0.5
    # one chunk (an interior one) against the float32 oracle: the chunked method is the reference's
    # own (RLdecon_large_in_memory.m:177-260 deconvolves each bordered chunk on its own)
    from oracle import decon as O
    ci = len(chunks) // 2 + 1
    c_host = chunks[ci].cpu().numpy().view(np.uint16).transpose(2, 1, 0)
    bx = boxes[ci]
    ref = O.decon_lucy_omw(np.asfortranarray(c_host), psf, bp, 2, background=100, bbox=bx, dtype=np.float32)
    got = outs[ci].cpu().numpy().view(np.uint16).transpose(2, 1, 0)
    chunk_lsb = int(np.max(np.abs(got.astype(np.int64) - ref.astype(np.int64))))
    chunk_rel = O.rel_l2(got.astype(np.float64), ref.astype(np.float64))
    _emit({"metric": "deconvolved Mvoxel/s (OMW, 2 iter), whole volume vs 512^3 chunks",
           "workload": "2048x2048x1024 uint16, 2M puncta (blurred puncta rendered directly: Gaussian PSF sigma 1.3/3.0), "
                       "31x31x41 PSF, OMW backprojector, OMW x2",
           "value": round(N / (whole_ms * 1e-3) / 1e6, 1), "unit": "Mvoxel/s", "ms_whole": round(whole_ms, 2),
           "chunked_value": round(N / (chunk_ms * 1e-3) / 1e6, 1), "ms_chunked": round(chunk_ms, 2),
           "chunks": n, "rel_l2_whole_vs_chunked": gap, "rel_l2_whole_vs_chunked_interior": gap_in,
           "chunk_vs_fp32_oracle": {"chunk": ci, "shape_yxz": list(c_host.shape), "uint16_rel_l2": chunk_rel,
                                    "max_lsb": chunk_lsb},
           "reference_cpu": "not run (the float32 CPU restatement needs ~100 GB of host RAM for this volume)"})


WORKLOADS = {"rl_small": wl_rl_small, "batched": wl_batched, "batched_passes": wl_batched_passes, "served": wl_served,
             "large": wl_large, "dsr": wl_dsr}

if __name__ == "__main__":
    main()
