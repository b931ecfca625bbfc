"""Benchmark of the grid ray-tracing hot path on B200.

Workload (one step): the 1,048,576-triangle "dense cluster in a sparse
field" scene held resident in HBM is rebuilt as a two-level grid (top
lambda = 1/16, leaf lambda = 4), then 1920x1080 primary closest-hit rays are
traced from a pinhole camera and 4 cosine-distributed ambient-occlusion
any-hit rays of length 0.1 are traced per primary hit (Philox seed 1).
The metric is Mrays/s over the whole step (build included); the build's
ms per million triangles is reported beside it.

  python bench.py [--gpus N --steps K --warmup W] [--impl reference]

Multi-GPU: replicas (every rank renders its own frame of the same scene, no
collective on the data path); value = all ranks' rays / max-over-ranks time.
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import threading
import time

from ctypes import byref as C_byref
from ctypes import c_void_p as C_void_p

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "Mrays/s"
N_TRIS = 1 << 20
AO_SPP, AO_LEN, AO_OFFSET, AO_SEED = 4, 0.1, 1e-4, 1
# direct illumination (DirectIlluminationIntegrator::shade): 4 shadow rays per hit to a
# 0.1 x 0.1 light 0.2 above the cluster, facing down
DI_SPP, DI_SEED = 4, 1
DI_LIGHT = dict(position=(-0.05, 0.2, -0.05), edge1=(0.1, 0.0, 0.0), edge2=(0.0, 0.0, 0.1),
                normal=(0.0, -1.0, 0.0), intensity=(10.0, 10.0, 10.0))
LAMBDA_TOP, LAMBDA_LEAF = 1.0 / 16.0, 4.0


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="shinobi", choices=["shinobi", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--cpu-sample-stride", type=int, default=64)
    ap.add_argument("--case", default="full", choices=["full", "small"],
                    help="small: 480x270 camera, for profiler captures (not a bench line)")
    ap.add_argument("--workload", default="cluster",
                    choices=["cluster", "direct", "batch", "serve", "pathtrace", "dynamic"],
                    help="cluster: the headline line; direct: the cluster frame shaded by an area light "
                         "(4 shadow rays per hit) instead of ambient occlusion; "
                         "batch: 256-scene batched vs one launch per scene; "
                         "serve: request stream with continuous batching vs one launch per request; "
                         "pathtrace: heightfield path tracer with compaction after every bounce; "
                         "dynamic: the cluster scene in motion (keyframe interpolation + rebuild of "
                         "frame N+1 overlapped with the render of frame N) against the sequential loop")
    ap.add_argument("--scenes", type=int, default=256, help="batch workload: number of scenes")
    ap.add_argument("--requests", type=int, default=20000, help="serve workload: requests per rate")
    ap.add_argument("--rates", default="1000,5000,20000,50000", help="serve workload: arrival rates (req/s)")
    ap.add_argument("--repeats", type=int, default=1, help="serve workload: runs per rate")
    ap.add_argument("--no-extras", action="store_true",
                    help="headline line only: skip the batched and served figures it carries at N=1")
    return ap.parse_args()


def workload_config(extra=None, direct=False):
    c = {"workload": "two-level grid rebuild + 1920x1080 primary + 4 AO rays/hit",
         "scene": "cluster_in_field: 1,048,576 tris (90% in r=0.05 sphere, offsets 0.002; 10% in [-50,50]^3, offsets 0.5), seed 1",
         "grid": "two-level, lambda_top=1/16 (divisor 1, min res 2), lambda_leaf=4, leaf threshold 16",
         "camera": "eye (0,0,-0.25), +z, 45 deg vertical FOV, 1920x1080, 1 spp",
         "ao": "4 cosine rays per hit, length 0.1, origin offset 1e-4, Philox4x32-10 seed 1",
         "l2": "flushed between timed steps (256 MiB write, outside the timed region)"}
    if direct:
        c["workload"] = "two-level grid rebuild + 1920x1080 primary + 4 area-light shadow rays/hit + shading"
        del c["ao"]
        c["direct"] = ("4 shadow segments per hit to a uniform point of the 0.1x0.1 light at y=0.2 "
                       "(normal -y, intensity 10), Philox4x32-10 seed 1; diffuse 0.7; frame + progressive final image")
    if extra:
        c.update(extra)
    return c


# ---------------------------------------------------------------------------
class ClockSampler:
    """SM clocks, power and clock-event (throttle) reasons sampled during the
    timed region: NVML polled every 2 ms from a thread, on the GPU this
    process runs on (found by its PCI bus id, whatever CUDA_VISIBLE_DEVICES
    says); one sample is taken at start and one at stop so a short region
    still has some.  Falls back to nvidia-smi when NVML is unavailable."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
    NAMES = ("hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap")

    def __init__(self, index: int):
        self.index = index
        self.proc = None
        self.nvml = None
        self.lines = []
        self.samples = []   # (sm MHz, reason bits)
        self.smax = None
        self.stop_flag = False

    def _nvml_handle(self):
        import pynvml
        import torch
        pynvml.nvmlInit()
        pr = torch.cuda.get_device_properties(self.index)
        bus = f"{pr.pci_domain_id:08X}:{pr.pci_bus_id:02X}:{pr.pci_device_id:02X}.0"
        return pynvml, pynvml.nvmlDeviceGetHandleByPciBusId(bus.encode())

    def _sample(self):
        nv, h = self.nvml
        self.samples.append((float(nv.nvmlDeviceGetClockInfo(h, nv.NVML_CLOCK_SM)),
                             int(nv.nvmlDeviceGetCurrentClocksEventReasons(h))))

    def _poll(self):
        while not self.stop_flag:
            try:
                self._sample()
            except Exception:
                return
            time.sleep(0.002)

    def start(self):
        try:
            self.nvml = self._nvml_handle()
            nv, h = self.nvml
            self.smax = float(nv.nvmlDeviceGetMaxClockInfo(h, nv.NVML_CLOCK_SM))
            self._sample()
            self.thread = threading.Thread(target=self._poll, daemon=True)
            self.thread.start()
            return
        except Exception:
            self.nvml = None
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.index), f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "100"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except Exception:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if self.nvml:
            self.stop_flag = True
            self.thread.join(timeout=5)
            try:
                self._sample()
            except Exception:
                pass
            nv, _ = self.nvml
            bits = {"hw_slowdown": nv.nvmlClocksEventReasonHwSlowdown,
                    "hw_thermal_slowdown": nv.nvmlClocksEventReasonHwThermalSlowdown,
                    "sw_thermal_slowdown": nv.nvmlClocksEventReasonSwThermalSlowdown,
                    "sw_power_cap": nv.nvmlClocksEventReasonSwPowerCap}
            reasons = {nm for nm, b in bits.items() for _, r in self.samples if r & b}
            sm = [c for c, _ in self.samples]
            return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": self.smax,
                    "reasons": sorted(reasons), "samples": len(sm), "source": "nvml"}
        if not self.proc:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        sm, smax, reasons = [], None, set()
        for ln in self.lines:
            parts = [p.strip() for p in ln.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                smax = float(parts[2])
            except ValueError:
                continue
            for nm, v in zip(self.NAMES, parts[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(nm)
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": smax,
                "reasons": sorted(reasons), "samples": len(sm), "source": "nvidia-smi"}


def measured_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            return json.load(f), "measured"
    return {"hbm_gbs": 6650.0, "bf16_tflops": 1590.0}, "fallback"


def fp32_peak_tflops(torch) -> float:
    """FP32 SIMT peak measured here: cuBLAS SGEMM (TF32 off), 8192^3, best of 5."""
    prev = torch.backends.cuda.matmul.allow_tf32
    torch.backends.cuda.matmul.allow_tf32 = False
    a = torch.randn(8192, 8192, device="cuda")
    b = torch.randn(8192, 8192, device="cuda")
    for _ in range(2):
        a @ b
    torch.cuda.synchronize()
    best = 1e9
    for _ in range(5):
        s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        s.record()
        a @ b
        e.record()
        torch.cuda.synchronize()
        best = min(best, s.elapsed_time(e))
    torch.backends.cuda.matmul.allow_tf32 = prev
    del a, b
    return 2.0 * 8192 ** 3 / (best * 1e-3) / 1e12


def profile_traffic():
    """DRAM bytes per launch of the dominant kernel from the committed ncu summary (or None)."""
    p = os.path.join(ROOT, "profiles", "traffic.json")
    if os.path.exists(p):
        with open(p) as f:
            return json.load(f)
    return {}


# ---------------------------------------------------------------------------
def cpu_baseline(sc, cam, stride: int, use_reference_build: bool, direct: bool = False):
    """Oracle port (or reference build + port traversal) on a bounded sample, host cores."""
    import oracle
    from shinobi_b200 import scenes  # noqa: F401
    threads = os.cpu_count() or 1
    oracle.set_threads(threads)
    b = oracle.bounds(sc.vertices, sc.indices)
    res = oracle.resolution(sc.num_triangles, b, LAMBDA_TOP, 1, 2)
    t0 = time.perf_counter()
    if use_reference_build:
        cells, leaves, refs = oracle.ref_host_build(sc.vertices, sc.indices, b, res)
        t_build = time.perf_counter() - t0
        g = oracle.grid_from_arrays(1, b, res, cells, leaves, refs, sc.vertices, sc.indices)
    else:
        g = oracle.build_two_level(sc.vertices, sc.indices, b, res, LAMBDA_LEAF, 16)
        t_build = time.perf_counter() - t0
    org, d = oracle.primary_rays(cam)
    sel = np.arange(0, org.shape[0], stride)
    t1 = time.perf_counter()
    tri, t, _, _, st_p = oracle.trace_closest(g, org[sel], d[sel])
    # the sample's secondary rays are keyed by their pixels' ids in the full
    # frame, so the sample's results are those of the frame at those pixels
    if direct:
        ro, rd, _ = oracle.direct_rays(org[sel], d[sel], tri, t, DI_SPP, DI_SEED, 0, DI_LIGHT, pix=sel)
        occ, st_s = oracle.trace_any(g, ro, rd, np.full(ro.shape[0], 0.9999, np.float32))
        shaded, _ = oracle.shade_direct(sc.vertices, sc.indices, org[sel], d[sel], tri, t, DI_SPP, DI_SEED, 0,
                                        DI_LIGHT, occ, pix=sel)
    else:
        ro, rd, rpix = oracle.ao_rays(sc.vertices, sc.indices, org[sel], d[sel], tri, t, AO_SPP, AO_SEED,
                                      AO_OFFSET, pix=sel)
        occ, st_s = oracle.trace_any(g, ro, rd, np.full(ro.shape[0], AO_LEN, np.float32))
        cnt = np.zeros(sel.size, np.int64)
        np.add.at(cnt, rpix, occ.astype(np.int64))
        shaded = np.where(tri == 0xFFFFFFFF, np.float32(1.0),
                          np.float32(1.0) - cnt.astype(np.float32) / np.float32(AO_SPP)).astype(np.float32)
    t_trace = time.perf_counter() - t1
    sample_rays = sel.size + ro.shape[0]
    # full-frame estimate: every pixel traced, AO rays in proportion to the sample's hit rate
    full_rays = org.shape[0] + ro.shape[0] * (org.shape[0] / sel.size)
    full_time = t_build + t_trace * (full_rays / sample_rays)
    return {
        "value": full_rays / full_time / 1e6, "unit": METRIC, "cores": threads,
        "kind": "reference" if use_reference_build else "port",
        "sample": (f"full grid build ({'reference TwoLevelGridBuilderHost::hostBuild, 1 thread' if use_reference_build else 'oracle two-level build, 1 thread'}, "
                   f"{t_build:.2f} s) + every {stride}th pixel's primary ray and its {'shadow rays and shading' if direct else 'AO rays'} "
                   f"({sample_rays} rays, {t_trace:.2f} s on {threads} threads), scaled to the full frame"),
        "build_ms_per_mtri": t_build * 1e3 / (sc.num_triangles / 1e6),
        "sample_seconds": t_build + t_trace,
        # the reference algorithm's work on the sample (oracle-counted cell visits
        # and triangle tests), scaled to the full frame by the sample ratio
        "oracle_work": {"scale": org.shape[0] / sel.size,
                        "primary": [int(st_p[0]), int(st_p[1])], "secondary": [int(st_s[0]), int(st_s[1])]},
        # the oracle's results on the sampled pixels (for the parity check of the timed frame)
        "oracle_sample": {"pixels": sel, "tri": tri, "t": t, "shaded": shaded},
    }


def frame_parity(sample, hits, shaded_dev, direct: bool):
    """The timed frame's results on the CPU baseline's sampled pixels against
    the oracle's (bit-exact: hit triangle, t and the AO value / shaded RGB)."""
    pix = sample["pixels"]
    tri = hits.tri.cpu().numpy().view(np.uint32)[pix]
    t = hits.t.cpu().numpy()[pix]
    if direct:
        got = shaded_dev.cpu().numpy().reshape(-1, 3)[pix]
    else:
        got = shaded_dev.cpu().numpy()[pix]
    bad_hit = int(np.count_nonzero((tri != sample["tri"]) | (t.view(np.uint32) != sample["t"].view(np.uint32))))
    ref = sample["shaded"]
    bad_sh = int(np.count_nonzero((got.view(np.uint32) != ref.view(np.uint32)).reshape(pix.size, -1).any(axis=1)))
    return {"pixels": int(pix.size), "mismatches": bad_hit + bad_sh, "hit_mismatches": bad_hit,
            ("shading_mismatches" if direct else "ao_mismatches"): bad_sh,
            "what": "the timed frame's primary hits (tri, t) and " + ("shaded RGB" if direct else "AO values")
                    + " on the CPU baseline's sampled pixels against the oracle, bit for bit"}


def run_reference(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    from shinobi_b200 import scenes
    sc = scenes.cluster_in_field(N_TRIS, seed=1)
    cam = scenes.CAMERA_CLUSTER
    # per-step sample sized so the whole run stays within a few minutes
    stride = max(64, 32 * (args.steps + args.warmup))
    direct = args.workload == "direct"
    for _ in range(args.warmup):
        cpu_baseline(sc, cam, stride * 4, True, direct=direct)
    vals, secs = [], 0.0
    last = None
    for _ in range(args.steps):
        last = cpu_baseline(sc, cam, stride, True, direct=direct)
        last.pop("oracle_sample")
        vals.append(last["value"])
        secs += last["sample_seconds"]
    v = float(np.mean(vals))
    line = {"impl": "reference", "metric": METRIC, "value": v, "unit": METRIC, "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": secs * 1e3 / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic (seeded Philox4x32-10 scene)",
            "config": workload_config(direct=direct),
            "cpu_baseline": {"value": v, "unit": METRIC, "cores": last["cores"], "kind": "reference",
                             "sample": last["sample"]},
            "build_ms_per_mtri": last["build_ms_per_mtri"],
            "e2e": {"value": v, "unit": METRIC, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


# ---------------------------------------------------------------------------
def max_over_ranks(x: float, dist, device="cuda") -> float:
    """Max of a per-rank scalar over all ranks (the identity on one rank).  The
    replicas share no data; this is the only collective of the bench."""
    if dist is None:
        return float(x)
    import torch
    t = torch.tensor([float(x)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def replica_value(world: int, units_per_rank: float, max_ms: float) -> float:
    """Whole-job throughput in millions of units/s: every rank processed
    units_per_rank, the job took the slowest rank's time."""
    return world * units_per_rank / (max_ms * 1e-3) / 1e6


def run_shinobi(args):
    import torch

    import shinobi_b200 as shn
    from shinobi_b200 import scenes

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime

        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                                device_id=torch.device("cuda", local))

    def barrier():
        if dist is not None:
            dist.barrier()

    ctx = shn.Context(local)
    sc = scenes.cluster_in_field(N_TRIS, seed=1)
    cam = scenes.CAMERA_CLUSTER
    if args.case == "small":
        cam = scenes.Camera(cam.eye, cam.forward, cam.up, cam.fov_deg, 480, 270)
        args.no_cpu_baseline = True
    npix = cam.res_x * cam.res_y
    stream = torch.cuda.current_stream()
    soup = shn.FaceSoup(sc.vertices, sc.indices, ctx=ctx)
    p = shn.grid_params(shn.SHN_GRID_TWO_LEVEL, lambda_=LAMBDA_TOP, top_divisor=1, min_res=2,
                        lambda_leaf=LAMBDA_LEAF, leaf_threshold=16)
    g = shn.Grid(ctx)
    hits = shn.alloc_hits(npix)
    direct = args.workload == "direct"
    ao = torch.empty(npix * (3 if direct else 1), dtype=torch.float32, device="cuda")
    final = torch.zeros(npix * 3, dtype=torch.float32, device="cuda") if direct else None
    dip = shn.di_params(light=DI_LIGHT, samples=DI_SPP, seed=DI_SEED) if direct else None
    nao = torch.zeros(1, dtype=torch.int32, device="cuda")

    def shade():
        if direct:
            g.shade_direct(cam, hits, dip, frame=ao, final=final, num_rays=nao)
        else:
            g.trace_ao(cam, hits, AO_SPP, AO_LEN, AO_OFFSET, AO_SEED, out=ao, num_rays=nao)
    flush = torch.empty(64 << 20, dtype=torch.int32, device="cuda")  # 256 MiB, twice the L2

    ev = lambda: torch.cuda.Event(enable_timing=True)  # noqa: E731

    def step(times=None):
        e0, e1, e2, e3 = ev(), ev(), ev(), ev()
        e0.record()
        g.build(soup, p)
        e1.record()
        g.trace_primary(cam, out=hits)
        e2.record()
        shade()
        e3.record()
        if times is not None:
            times.append((e0, e1, e2, e3))

    for _ in range(max(3, args.warmup)):
        step()
    torch.cuda.synchronize()
    n_ao = int(nao.item())
    rays_per_step = npix + n_ao

    # ---- device-timed region (inputs resident in HBM) -------------------------
    clocks = ClockSampler(local)
    clocks.start()
    barrier()
    torch.cuda.synchronize()
    times = []
    for _ in range(args.steps):
        flush.fill_(1)          # L2 flush, outside the step's events
        step(times)
    torch.cuda.synchronize()
    barrier()
    clk = clocks.stop()
    per = np.array([[a.elapsed_time(b), b.elapsed_time(c), c.elapsed_time(d)] for a, b, c, d in times])
    step_ms = per.sum(axis=1)
    total_ms = float(step_ms.sum())
    total_ms = max_over_ranks(total_ms, dist)
    value = replica_value(world, args.steps * rays_per_step, total_ms)
    build_ms = float(per[:, 0].mean())
    prim_ms = float(per[:, 1].mean())
    ao_ms = float(per[:, 2].mean())

    # ---- end to end through the C ABI with host buffers ------------------------
    # Every step uploads its geometry from pinned host memory and reads its
    # hits and shading back into pinned host memory.  The copies run on two
    # copy streams, pipelined with the compute stream: step k+1's vertices
    # upload and step k's results download while the GPU computes, with
    # double-buffered device inputs and outputs.  The timed region runs from
    # the first upload to the last download; every byte of every step is in it.
    hv = torch.from_numpy(sc.vertices).pin_memory()
    dv = [torch.empty(hv.shape, dtype=hv.dtype, device="cuda") for _ in range(2)]
    hits_b = [hits, shn.alloc_hits(npix)]
    ao_b = [ao, torch.empty_like(ao)]
    final_b = [final, final]      # the progressive image: one buffer, each step blends into it
    h_tri = [torch.empty(npix, dtype=torch.int32).pin_memory() for _ in range(2)]
    h_t = [torch.empty(npix, dtype=torch.float32).pin_memory() for _ in range(2)]
    h_ao = [torch.empty(ao.numel(), dtype=torch.float32).pin_memory() for _ in range(2)]
    comp = torch.cuda.current_stream()
    up, down = torch.cuda.Stream(), torch.cuda.Stream()
    ev_in = [torch.cuda.Event() for _ in range(2)]     # vertices of buffer b uploaded
    ev_used = [torch.cuda.Event() for _ in range(2)]   # vertices of buffer b consumed by the scene
    ev_done = [torch.cuda.Event() for _ in range(2)]   # results of buffer b written
    ev_read = [torch.cuda.Event() for _ in range(2)]   # results of buffer b copied to the host

    def e2e_run(nsteps):
        up.wait_stream(comp)                            # after the start event
        with torch.cuda.stream(up):
            dv[0].copy_(hv, non_blocking=True)
            ev_in[0].record(up)
        for k in range(nsteps):
            b = k & 1
            if k + 1 < nsteps:                          # next step's geometry, ahead of time
                with torch.cuda.stream(up):
                    if k >= 1:
                        up.wait_event(ev_used[1 - b])
                    dv[1 - b].copy_(hv, non_blocking=True)
                    ev_in[1 - b].record(up)
            flush.fill_(1)                              # L2 flush between steps
            comp.wait_event(ev_in[b])
            if k >= 2:
                comp.wait_event(ev_read[b])             # buffer b's last results are on the host
            soup.update_vertices(dv[b])                 # the step's geometry into the scene
            ev_used[b].record(comp)
            g.build(soup, p)
            g.trace_primary(cam, out=hits_b[b])
            if direct:
                g.shade_direct(cam, hits_b[b], dip, frame=ao_b[b], final=final_b[b], num_rays=nao)
            else:
                g.trace_ao(cam, hits_b[b], AO_SPP, AO_LEN, AO_OFFSET, AO_SEED, out=ao_b[b], num_rays=nao)
            ev_done[b].record(comp)
            with torch.cuda.stream(down):               # the step's results to the host
                down.wait_event(ev_done[b])
                h_tri[b].copy_(hits_b[b].tri, non_blocking=True)
                h_t[b].copy_(hits_b[b].t, non_blocking=True)
                h_ao[b].copy_(ao_b[b], non_blocking=True)
                ev_read[b].record(down)
        comp.wait_stream(down)

    e2e_run(2)
    torch.cuda.synchronize()
    barrier()
    e_s, e_e = ev(), ev()
    e_s.record()
    e2e_run(args.steps)
    e_e.record()
    torch.cuda.synchronize()
    e2e_total = max_over_ranks(e_s.elapsed_time(e_e), dist)
    e2e_value = replica_value(world, args.steps * rays_per_step, e2e_total)
    h2d = int(sc.vertices.nbytes)
    d2h = int(npix * 8 + ao.numel() * 4)
    assert np.array_equal(h_tri[(args.steps - 1) & 1].numpy(), hits_b[(args.steps - 1) & 1].tri.cpu().numpy())

    # ---- roofline of the dominant kernel (work counters, untimed pass) ---------
    cnt = torch.zeros(2, dtype=torch.int64, device="cuda")
    ctx.lib.shn_grid_set_stats(g.handle, shn._ptr(cnt))
    cnt.zero_()
    g.trace_primary(cam, out=hits)
    torch.cuda.synchronize()
    prim_steps, prim_tests = [int(x) for x in cnt.cpu().tolist()]
    cnt.zero_()
    shade()
    torch.cuda.synchronize()
    ao_steps, ao_tests = [int(x) for x in cnt.cpu().tolist()]
    ctx.lib.shn_grid_set_stats(g.handle, None)
    fp32 = fp32_peak_tflops(torch)
    cpu = None
    parity = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        # the GPU results of the last step (the same scene, camera and seeds every step)
        step()
        torch.cuda.synchronize()
        g.sync_status()
        cpu = cpu_baseline(sc, cam, args.cpu_sample_stride, False, direct=direct)
        parity = frame_parity(cpu.pop("oracle_sample"), hits, ao, direct)
    # dominant kernel: the longer of the two trace kernels
    if ao_ms >= prim_ms:
        kname = "k_trace_direct<two-level>" if direct else "k_trace_ao<two-level>"
        kms, ksteps, ktests = ao_ms, ao_steps, ao_tests
    else:
        kname, kms, ksteps, ktests = "k_trace_camera<two-level>", prim_ms, prim_steps, prim_tests
    # executed work (device counters): block culling skips most of the tests
    # the reference algorithm makes
    work = 10.0 * ksteps + 40.0 * ktests  # FP32 ops per launch (cell visit 10, triangle test 40)
    executed = work / (kms * 1e-3) / 1e12
    algorithmic = None
    if cpu is not None:
        # the reference algorithm's work (no block culling): what the kernel
        # would execute without skipping blocks, as a rate -- above the FP32
        # peak, so reported beside the roofline, not as its fraction
        ow = cpu.pop("oracle_work")
        which = "primary" if kname.startswith("k_trace_camera") else "secondary"
        a_steps, a_tests = (ow[which][0] * ow["scale"], ow[which][1] * ow["scale"])
        arate = (10.0 * a_steps + 40.0 * a_tests) / (kms * 1e-3) / 1e12
        algorithmic = {"tflops": arate, "vs_peak": arate / fp32,
                       "work": (f"{a_steps:.4g} cell visits x 10 + {a_tests:.4g} triangle tests x 40 FP32 ops per "
                                f"launch: the reference algorithm's work, counted by the oracle on every "
                                f"{args.cpu_sample_stride}th pixel and scaled to the frame")}
    traffic = profile_traffic().get(kname)
    inf = g.info()
    peaks, peak_kind = measured_peaks()
    # build bytes (algorithmic): geometry 2 passes + emit + sort + ranges, both levels
    P, R, L = int(inf.num_top_refs), int(inf.num_refs), int(inf.num_leaves)
    C0 = int(inf.num_cells)

    def sort_bytes(k, bits):
        return 8 * k * (1 + 2 * ((bits + 7) // 8))

    b_build = (96 * N_TRIS + 8 * P + sort_bytes(P, max(1, (C0 - 1).bit_length())) + 12 * P + 8 * C0
               + 48 * P + 8 * R + sort_bytes(R, max(1, (L - 1).bit_length())) + 12 * R + 8 * L + 4 * C0
               + 48 * R)
    build_gbs = b_build / (build_ms * 1e-3) / 1e9

    line = {
        "metric": METRIC, "value": value, "unit": METRIC, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": total_ms / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic (seeded Philox4x32-10 scene, resident in HBM)",
        "config": workload_config(direct=direct),
        "rays_per_step": rays_per_step, "parallelism": f"replicas x{world}",
        "build_ms_per_mtri": build_ms / (N_TRIS / 1e6),
        "phase_ms": {"build": build_ms, "primary": prim_ms, ("direct" if direct else "ao"): ao_ms},
        "e2e": {"value": e2e_value, "unit": METRIC, "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h,
                "ms_per_step": e2e_total / args.steps,
                "what": "shn_scene_update_vertices + shn_grid_build + shn_trace_primary + shading per step, "
                        "vertices uploaded from and hits + shading read back to pinned host memory every step "
                        "on two copy streams pipelined with the compute stream (double-buffered)"},
        "roofline": {
            "bound": "fp32", "kernel": kname, "achieved": executed, "peak": fp32, "unit": "TFLOP/s",
            "frac": executed / fp32, "traffic": traffic,
            "work": (f"{ksteps} cell visits x 10 + {ktests} triangle tests x 40 FP32 ops per launch as executed "
                     "(device counters of the kernel's counting variant)"),
            "peak_source": "cuBLAS SGEMM (TF32 off) 8192^3 measured in this run; no FP32 figure in MEASURED_PEAKS.json",
            "algorithmic_rate": algorithmic,
        },
        "roofline_build": {
            "bound": "hbm", "achieved": build_gbs, "peak": peaks["hbm_gbs"], "unit": "GB/s",
            "frac": build_gbs / peaks["hbm_gbs"], "traffic": None,
            "note": f"whole two-level build (all kernels) per step; peak {peak_kind}",
        },
        "clocks": clk,
    }
    # kernels launched per step: build (uniform count+emit+sort+ranges, leaf stage) + primary + AO (compact, trace, finalize)
    line["gpu_launches"] = args.steps * launches_per_step(P, R, C0, L)
    if cpu is not None:
        line["cpu_baseline"] = cpu
        line["parity"] = parity
    if rank == 0 and world == 1 and not args.no_extras and args.case == "full":
        # the batched (256 scenes) and served (64 resident scenes) forms beside
        # the headline, each against its plain one-launch-per-request path
        del soup, g, hits, ao, final, flush, cnt
        ctx.close()                 # the context's memory pool goes with its last object
        torch.cuda.synchronize()
        torch.cuda.empty_cache()
        line["batch"] = batch_summary(run_batch(sub_args(args, steps=min(args.steps, 5), warmup=2), emit=False))
        torch.cuda.empty_cache()
        line["serve"] = serve_summary(run_serve(sub_args(args, requests=5000, rates="5000,50000", repeats=2),
                                                emit=False))
    if rank == 0:
        print(json.dumps(line), flush=True)
    if dist is not None:
        dist.destroy_process_group()


def sub_args(args, **kw):
    a = argparse.Namespace(**vars(args))
    for k, v in kw.items():
        setattr(a, k, v)
    return a


def batch_summary(b):
    return {"workload": b["config"]["workload"], "value": b["value"], "unit": METRIC, "ms_per_step": b["ms_per_step"],
            "plain_value": b["plain"]["value"], "plain_ms_per_step": b["plain"]["ms_per_step"],
            "batched_vs_plain": b["batched_vs_plain"], "results_identical_to_plain": b["results_identical_to_plain"],
            "build_ms": b["build_ms"], "build_hbm_frac": b["roofline_build"]["frac"],
            "step": b["config"]["step"], "steps": b["steps"]}


def serve_summary(sv):
    out = {"workload": sv["config"]["workload"], "unit": METRIC, "rates": {}}
    for r in sv["config"]["rates_req_per_s"]:
        c, p = sv["served"]["coalesced"][r], sv["served"]["plain"][r]
        out["rates"][r] = {
            "coalesced": {k: c[k] for k in ("mrays_per_s", "p50_ms", "p99_ms", "runs")},
            "plain": {k: p[k] for k in ("mrays_per_s", "p50_ms", "p99_ms", "runs")},
            "mrays_ratio": sv["speedup_at_rate"][r], "p99_ratio": sv["p99_ratio_at_rate"][r]}
    return out


def launches_per_step(P, R, C0, L):
    def sort_launches(n, cells):
        # the emission counts the digits: a digit-offset scan + one launch per
        # 8- or 9-bit pass (whichever takes fewer passes)
        if n <= 1:
            return 0
        bits = max(1, (cells - 1).bit_length())
        p8, p9 = (bits + 7) // 8, (bits + 8) // 9
        return 1 + min(p8, p9)
    build = (2 + 1 + sort_launches(P, C0) + 1      # count + scan, emit, sort, top ranges
             + 1 + 2 + 1 + sort_launches(R, L) + 1)  # leaf cells scan, leaf count + scan, emit, sort, ranges
    # Morton order of the triangles (keys, two 4-pass sorts, second keys, permute)
    # and the boxes per 32 and per 1024 references
    spatial = 1 + 2 * (2 + 4) + 1 + 1 + (2 if R else 0) + 3   # + the three leaf-distance passes
    return build + spatial + 1 + 3                     # primary; compact + trace + finalize (AO or shading)


def run_batch(args, emit=True):
    """Batched multi-scene build + trace (one fused pipeline and one launch, captured in a CUDA
    graph, autotuned lambda) against the plain path (one build + one trace launch per scene)."""
    import torch

    import shinobi_b200 as shn
    from shinobi_b200 import scenes

    torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", "0")))
    ns = args.scenes
    tris, scales, rays = scenes.batch_workload_sizes(ns)
    # scenes generated on the GPU and concatenated (indices local to each scene)
    vs, ix = [], []
    for i in range(ns):
        v, t = scenes.uniform_soup_device(int(tris[i]), seed=1000 + i, offset_scale=float(scales[i]))
        vs.append(v)
        ix.append(t)
    vo = np.concatenate([[0], np.cumsum(3 * tris)]).astype(np.uint32)
    to = np.concatenate([[0], np.cumsum(tris)]).astype(np.uint32)
    V = torch.cat(vs)
    I = torch.cat(ix)
    del vs, ix
    ro = np.concatenate([[0], np.cumsum(rays)]).astype(np.uint32)
    orgs, dirs = [], []
    for i in range(ns):
        o, d = scenes.random_rays_device(int(rays[i]), seed=77, stream=i)
        orgs.append(o)
        dirs.append(d)
    org = torch.cat(orgs)
    dirs_t = torch.cat(dirs)
    del orgs, dirs
    n_rays = int(ro[-1])
    n_tris = int(to[-1])
    # a context of its own: its memory pool is released with the last object
    # of the batch when this function returns
    ctx = shn.Context(int(os.environ.get("LOCAL_RANK", "0")))
    lib = ctx.lib
    h = C_void_p()
    ctx.check(lib.shn_batch_create(ctx.handle, ns, shn._ptr(V), vo.ctypes.data_as(C_void_p), shn._ptr(I),
                                   to.ctypes.data_as(C_void_p), 1, shn._stream(None), C_byref(h)),
              "shn_batch_create")
    bt = shn.Batch.__new__(shn.Batch)
    bt.ctx, bt.handle, bt.num_scenes, bt.tri_offsets = ctx, h, ns, to
    t0 = time.perf_counter()
    cands = np.array([0.5, 0.75, 1.0, 1.5, 2.0, 3.0], np.float32)
    chosen, chosen_sah, tune_report = bt.autotune_ex(cands, expected_rays=rays.astype(np.uint32),
                                                     sample_rays=16384, blocks_per_sm=(0, 4, 6),
                                                     sort_tiles=(6144, 4096))
    t_tune = time.perf_counter() - t0
    bt.build()
    torch.cuda.synchronize()
    build_times = []
    for _ in range(3):
        bt.build()
        build_times.append(bt.info()["build_ms"])
    info = bt.info()
    out = shn.alloc_hits(n_rays, uv=False)
    bt.capture(org, dirs_t, ro, out)
    for _ in range(max(2, args.warmup)):
        bt.replay()
    torch.cuda.synchronize()
    ev = lambda: torch.cuda.Event(enable_timing=True)  # noqa: E731
    ms = []
    for _ in range(args.steps):
        a, b = ev(), ev()
        torch.cuda.nvtx.range_push("shn_batch_step")   # profiler filter: --nvtx-include shn_batch_step/
        a.record()
        bt.replay()
        b.record()
        torch.cuda.nvtx.range_pop()
        torch.cuda.synchronize()
        ms.append(a.elapsed_time(b))
    batched_ms = float(np.mean(ms))
    batched = n_rays / (batched_ms * 1e-3) / 1e6
    # plain: one build + one trace launch per scene (the per-request path)
    grid = shn.Grid(ctx)
    soups = []
    for i in range(ns):
        soups.append(shn.FaceSoup(V[vo[i]:vo[i + 1]], I[to[i]:to[i + 1]], ctx=ctx))
    hits = shn.alloc_hits(n_rays, uv=False)
    cols = [org[:, k].contiguous() for k in range(3)] + [dirs_t[:, k].contiguous() for k in range(3)]

    def plain_once():
        for i in range(ns):
            p = shn.grid_params(shn.SHN_GRID_UNIFORM, lambda_=float(chosen[i]))
            grid.build(soups[i], p)
            a, b = int(ro[i]), int(ro[i + 1])
            r = shn._abi.Rays(*[shn._ptr(c[a:b]) for c in cols], None)
            hh = shn._abi.Hits(shn._ptr(hits.tri[a:b]), shn._ptr(hits.t[a:b]), None, None)
            ctx.check(lib.shn_trace_closest(grid.handle, C_byref(r), b - a, C_byref(hh), shn._stream(None)),
                      "plain trace")

    plain_once()
    torch.cuda.synchronize()
    pms = []
    for _ in range(max(1, min(args.steps, 3))):
        a, b = ev(), ev()
        a.record()
        plain_once()
        b.record()
        torch.cuda.synchronize()
        pms.append(a.elapsed_time(b))
    plain_ms = float(np.mean(pms))
    plain = n_rays / (plain_ms * 1e-3) / 1e6
    same = bool(torch.equal(hits.tri, out.tri))
    peaks, peak_kind = measured_peaks()
    P, Ct = int(info["num_pairs"]), int(info["total_cells"])
    bits = max(1, (Ct - 1).bit_length())
    # geometry two passes, emit, sort, ranges + indices (the batch keeps no reference-ordered copy)
    b_build = 96 * n_tris + 8 * P + 8 * P * (1 + 2 * ((bits + 7) // 8)) + 12 * P + 8 * Ct
    bms = float(np.median(build_times))
    line = {
        "metric": METRIC, "value": batched, "unit": METRIC, "n_gpus": 1, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": batched_ms, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded Philox4x32-10 scenes, generated on the GPU)",
        "config": {"workload": f"batched: {ns} scenes, {n_tris} tris (log-U[1K,2M]/scene, offset scale log-U[0.001,0.05]), "
                               f"{n_rays} random rays (log-U[64K,1M]/scene), uniform grids, closest hit",
                   "step": "CUDA graph replay of the fused batched build + one trace launch",
                   "lambda_candidates": cands.tolist(),
                   "lambda_chosen_histogram": {str(c): int((chosen == c).sum()) for c in cands}},
        "plain": {"value": plain, "unit": METRIC, "ms_per_step": plain_ms,
                  "what": "one shn_grid_build + one shn_trace_closest launch per scene, same lambdas"},
        "batched_vs_plain": batched / plain,
        "results_identical_to_plain": same,
        "build_ms": bms, "build_ms_per_mtri": bms / (n_tris / 1e6), "autotune_s": t_tune,
        "autotune": {"timed_candidates": tune_report["timed_candidates"],
                     "trace_blocks_per_sm": tune_report["blocks_per_sm"],
                     "shape_ms": dict(zip(("occupancy", "4", "6"), tune_report["shape_ms"])),
                     "sort_tile_keys": tune_report["sort_tile_keys"],
                     "sort_tile_build_ms": dict(zip(("6144", "4096"), tune_report["sort_tile_ms"])),
                     "sah_cost_chosen_median": float(np.median(chosen_sah))},
        "roofline_build": {"bound": "hbm", "achieved": b_build / (bms * 1e-3) / 1e9, "peak": peaks["hbm_gbs"],
                           "unit": "GB/s", "frac": b_build / (bms * 1e-3) / 1e9 / peaks["hbm_gbs"],
                           "traffic": None, "note": f"whole batched build, algorithmic bytes {b_build}; peak {peak_kind}"},
    }
    bt.close()
    if emit:
        print(json.dumps(line), flush=True)
    return line


def run_pathtrace(args):
    """Plain path tracer on the heightfield scene: 2048x1024 quads (Perlin height, seed 2, amplitude
    0.1) + 1000 boxes, uniform grid lambda=5, 1920x1080 x 16 spp, depth 4, roulette from depth 2,
    albedo 0.7, one area light, compaction after every bounce.  A step is one full render."""
    import torch

    import shinobi_b200 as shn
    from shinobi_b200 import scenes

    torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", "0")))
    sc = scenes.heightfield_boxes(2048, 1024, nboxes=1000)
    soup = shn.FaceSoup(sc.vertices, sc.indices)
    grid = shn.Grid()
    p = shn.grid_params(shn.SHN_GRID_UNIFORM, lambda_=5.0)
    for _ in range(2):
        grid.build(soup, p)
    build_ms = float(np.median([grid.build(soup, p).info().build_ms for _ in range(3)]))
    cam = scenes.CAMERA_HEIGHTFIELD
    small = args.case == "small"
    if small:
        cam = scenes.Camera(cam.eye, cam.forward, cam.up, cam.fov_deg, 480, 270)
    spp = 4 if small else 16
    params = shn.pt_params(spp=spp, max_depth=4, rr_depth=2, albedo=0.7, seed=2)
    stats = torch.zeros(params.max_depth + 1, dtype=torch.int32, device="cuda")
    img = torch.empty(cam.res_x * cam.res_y * 3, dtype=torch.float32, device="cuda")
    for _ in range(max(1, args.warmup)):
        grid.pt_render(soup, cam, params, out=img)
    torch.cuda.synchronize()
    ev = lambda: torch.cuda.Event(enable_timing=True)  # noqa: E731
    clocks = ClockSampler(torch.cuda.current_device())
    clocks.start()
    ms = []
    for _ in range(args.steps):
        stats.zero_()
        a, b = ev(), ev()
        torch.cuda.nvtx.range_push("shn_pathtrace_step")
        a.record()
        grid.pt_render(soup, cam, params, out=img, stats=stats)
        b.record()
        torch.cuda.nvtx.range_pop()
        torch.cuda.synchronize()
        ms.append(a.elapsed_time(b))
    clk = clocks.stop()
    st = stats.cpu().numpy().astype(np.int64)
    ext, shadow = int(st[:params.max_depth].sum()), int(st[params.max_depth])
    rays = ext + shadow
    step_ms = float(np.mean(ms))
    # end to end: the scene's vertices from pinned host memory, the render, the image back
    vtx_h = torch.from_numpy(np.ascontiguousarray(sc.vertices)).pin_memory()
    vtx_d = torch.empty_like(vtx_h, device="cuda")
    img_h = torch.empty(img.numel(), dtype=torch.float32).pin_memory()
    e2e = []
    for _ in range(max(1, min(args.steps, 3))):
        a, b = ev(), ev()
        a.record()
        vtx_d.copy_(vtx_h, non_blocking=True)
        soup.update_vertices(vtx_d)
        grid.build(soup, p)
        grid.pt_render(soup, cam, params, out=img)
        img_h.copy_(img, non_blocking=True)
        b.record()
        torch.cuda.synchronize()
        e2e.append(a.elapsed_time(b))
    e2e_ms = float(np.mean(e2e))
    line = {
        "metric": METRIC, "value": rays / (step_ms * 1e-3) / 1e6, "unit": METRIC, "n_gpus": 1,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": step_ms, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic (seeded Perlin heightfield + lognormal boxes, resident in HBM)",
        "config": {"workload": f"path tracer: {sc.num_triangles} tris (2048x1024 heightfield quads + 1000 boxes), "
                               f"uniform grid lambda=5, {cam.res_x}x{cam.res_y} x {spp} spp, depth 4, "
                               "roulette from depth 2, albedo 0.7, one area light, compaction after every bounce",
                   "rays_per_step": rays, "extension_rays": ext, "shadow_rays": shadow,
                   "paths_per_bounce": st[:params.max_depth].tolist(),
                   "l2": "inputs larger than L2 (paths: 64 B x 33M per bounce)"},
        "build_ms_per_mtri": build_ms / (sc.num_triangles / 1e6),
        "e2e": {"value": rays / (e2e_ms * 1e-3) / 1e6, "unit": METRIC,
                "h2d_bytes_per_step": int(vtx_h.numel() * 4), "d2h_bytes_per_step": int(img_h.numel() * 4),
                "what": "vertex upload from pinned host memory + rebuild + render + image read-back"},
        "clocks": clk,
    }
    print(json.dumps(line), flush=True)


def run_serve(args, emit=True):
    """Served ray-query stream: 64 resident scenes, Poisson arrivals, closest/any mix, 2% updates."""
    import torch

    import shinobi_b200 as shn
    from shinobi_b200 import scenes

    torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", "0")))
    ns = 64
    tris, scales, _ = scenes.batch_workload_sizes(ns, seed=11)
    scs = []
    for i in range(ns):
        v, t = scenes.uniform_soup_device(int(tris[i]), seed=2000 + i, offset_scale=float(scales[i]))
        scs.append(scenes.Scene(v.cpu().numpy(), t.cpu().numpy().astype(np.uint32)))
    repl = []
    for k in range(8):   # replacement scenes (new seeds) for the update requests
        i = k % ns
        v, t = scenes.uniform_soup_device(int(tris[i]), seed=9000 + k, offset_scale=float(scales[i]))
        repl.append((i, scenes.Scene(v.cpu().numpy(), t.cpu().numpy().astype(np.uint32))))
    pool_n = 8 << 20
    o, d = scenes.random_rays_device(pool_n, seed=55)
    pool = torch.zeros(pool_n, 8, dtype=torch.float32)
    pool[:, 0:3] = o.cpu()
    pool[:, 3:6] = d.cpu()
    pool[:, 6] = 1e30
    pool = pool.pin_memory()
    any_pool = pool.clone().pin_memory()
    any_pool[:, 6] = 0.1
    out_tri = torch.empty(pool_n, dtype=torch.int32).pin_memory()
    out_t = torch.empty(pool_n, dtype=torch.float32).pin_memory()
    rng = np.random.default_rng(99)
    n_req = args.requests
    counts = np.floor(np.exp(rng.uniform(np.log(1e3), np.log(1e6), n_req))).astype(np.int64)
    kinds = (rng.random(n_req) < 0.5).astype(np.int64)
    slots = rng.integers(0, ns, n_req)
    is_upd = rng.random(n_req) < 0.02
    starts = np.array([rng.integers(0, pool_n - c) for c in counts], np.int64)
    budget = 120 << 30
    results = {}
    for coalesce in (True, False):
        ctx = shn.Context(0, hbm_budget_bytes=budget)
        srv = shn.Server(ctx=ctx, num_slots=ns, coalesce=coalesce)
        for i, sc in enumerate(scs):
            srv.load_scene(i, sc)
        reqs = []
        upd_k = 0
        for k in range(n_req):
            if is_upd[k]:
                slot, sc = repl[upd_k % len(repl)]
                upd_k += 1
                reqs.append(srv.update_request(slot, sc))
                continue
            src = pool if kinds[k] == 0 else any_pool
            a, c = int(starts[k]), int(counts[k])
            r = shn._abi.Request()
            r.kind, r.scene, r.num_rays = int(kinds[k]), int(slots[k]), c
            r.rays = C_void_p(src.data_ptr() + 32 * a)
            r.out_tri = C_void_p(out_tri.data_ptr() + 4 * a)
            r.out_t = C_void_p(out_t.data_ptr() + 4 * a)
            reqs.append(r)
        # warm-up: a short schedule with updates (first launches of every kernel, pool growth)
        wn = min(400, n_req)
        srv.run_schedule(reqs[:wn], np.arange(wn, dtype=np.float64) * 1e-4)
        srv.drain()
        per_rate = {}
        for rate in [float(x) for x in args.rates.split(",")]:
            runs = []
            for rep_i in range(max(1, getattr(args, "repeats", 1))):
                gaps = np.random.default_rng(1000 * rep_i + int(rate)).exponential(1.0 / rate, n_req)
                arr = np.cumsum(gaps) - gaps[0]
                srv.stats(reset=True)
                res = srv.run_schedule(reqs, arr)
                rec = srv.records()
                st = srv.stats(reset=True)
                q_lat = rec["latency_us"][rec["kind"] != shn._abi.SHN_REQ_UPDATE] / 1e3
                u_lat = rec["latency_us"][rec["kind"] == shn._abi.SHN_REQ_UPDATE] / 1e3
                runs.append({"p50_ms": st["p50_us"] / 1e3, "p99_ms": st["p99_us"] / 1e3,
                             "mrays_per_s": st["mrays_per_s"], "launches": st["launches"],
                             "requests": st["requests"], "failed": int((res != 0).sum()),
                             "wall_s": st["wall_s"], "offered_mrays_per_s": float(counts[~is_upd].sum()) / arr[-1] / 1e6,
                             "query_p50_ms": float(np.percentile(q_lat, 50)) if q_lat.size else None,
                             "query_p99_ms": float(np.percentile(q_lat, 99)) if q_lat.size else None,
                             "update_p50_ms": float(np.percentile(u_lat, 50)) if u_lat.size else None,
                             "update_p99_ms": float(np.percentile(u_lat, 99)) if u_lat.size else None})
            # the mean over the runs, and every run for the spread between them
            agg = {k: float(np.mean([r[k] for r in runs if r[k] is not None])) if any(r[k] is not None for r in runs)
                   else None for k in runs[0]}
            agg["runs"] = [{k: r[k] for k in ("mrays_per_s", "p50_ms", "p99_ms")} for r in runs]
            per_rate[str(int(rate))] = agg
        results["coalesced" if coalesce else "plain"] = per_rate
        srv.close()
        ctx.close()
    rates = list(results["coalesced"].keys())
    top = rates[-1]
    line = {
        "metric": METRIC, "value": results["coalesced"][top]["mrays_per_s"], "unit": METRIC, "n_gpus": 1,
        "steps": 1, "warmup": 0, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f32", "data": "synthetic (seeded scenes and ray pool)",
        "config": {"workload": f"served: {ns} resident scenes ({int(tris.sum())} tris), {n_req} requests per rate, "
                               "rays log-U[1K,1M] from a pinned pool, closest/any p=0.5 (any: length 0.1), "
                               "2% scene replacements (device rebuild), HBM budget 120 GB",
                   "rates_req_per_s": rates},
        "served": results,
        "speedup_at_rate": {r: results["coalesced"][r]["mrays_per_s"] / max(1e-9, results["plain"][r]["mrays_per_s"]) for r in rates},
        "p99_ratio_at_rate": {r: results["coalesced"][r]["p99_ms"] / max(1e-9, results["plain"][r]["p99_ms"]) for r in rates},
    }
    if emit:
        print(json.dumps(line), flush=True)
    return line


def run_dynamic(args):
    """DynamicRTEngine: every frame interpolates the 1M-triangle cluster scene
    between two keyframes and rebuilds its two-level grid while the previous
    frame's grid renders (1920x1080 primary + 4 area-light shadow rays per
    hit + shading), against the sequential interpolate -> rebuild -> render."""
    import torch

    import shinobi_b200 as shn
    from shinobi_b200 import scenes

    torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", "0")))
    sc = scenes.cluster_in_field(N_TRIS, seed=1)
    base = sc.vertices
    move = scenes.uniform_draws(base.shape[0], 3, 7, scenes.TAG_RAYS)
    kf2 = (base + (move - np.float32(0.5)) * np.float32(0.002)).astype(np.float32)
    kf1_t = torch.from_numpy(base).cuda()
    kf2_t = torch.from_numpy(kf2).cuda()
    p = shn.grid_params(shn.SHN_GRID_TWO_LEVEL, lambda_=LAMBDA_TOP, top_divisor=1, min_res=2,
                        lambda_leaf=LAMBDA_LEAF, leaf_threshold=16)
    cam = scenes.CAMERA_CLUSTER
    npix = cam.res_x * cam.res_y
    di = shn.di_params(light=DI_LIGHT, samples=DI_SPP, seed=DI_SEED)
    hits = shn.alloc_hits(npix)
    frame = torch.empty(cam.res_y, cam.res_x, 3, dtype=torch.float32, device="cuda")
    eng = shn.DynamicEngine(base, sc.indices, p)
    coeff = lambda k: 0.5 + 0.5 * np.sin(0.3 * k)  # noqa: E731
    for k in range(max(3, args.warmup)):
        eng.render_frame(kf1_t, kf2_t, coeff(k), cam, di, hits, frame)
    dyn, rays = [], 0
    clocks = ClockSampler(torch.cuda.current_device())
    clocks.start()
    for k in range(args.steps):
        r_ms, b_ms, f_ms = eng.render_frame(kf1_t, kf2_t, coeff(k + args.warmup), cam, di, hits, frame)
        dyn.append((r_ms, b_ms, f_ms))
        rays += npix + DI_SPP * int((hits.tri != -1).sum().item())
    clk = clocks.stop()
    eng.close()
    dyn = np.array(dyn)
    # sequential: one stream, interpolate + rebuild + render per frame
    soup = shn.FaceSoup(base, sc.indices)
    g = shn.Grid()
    ev = lambda: torch.cuda.Event(enable_timing=True)  # noqa: E731
    seq = []
    for k in range(max(3, args.warmup) + args.steps):
        a, b = ev(), ev()
        a.record()
        soup.interpolate_vertices(kf1_t, kf2_t, coeff(k))
        g.build(soup, p)
        h = g.trace_primary(cam, out=hits)
        g.shade_direct(cam, h, di, frame=frame)
        b.record()
        torch.cuda.synchronize()
        if k >= max(3, args.warmup):
            seq.append(a.elapsed_time(b))
    seq_ms = float(np.mean(seq))
    f_ms = float(dyn[:, 2].mean())
    line = {
        "metric": METRIC, "value": rays / (dyn[:, 2].sum() * 1e-3) / 1e6, "unit": METRIC, "n_gpus": 1,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": f_ms, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic (seeded Philox4x32-10 scene and keyframe motion, resident in HBM)",
        "config": {"workload": "dynamic: 1,048,576-tri cluster scene between two keyframes (motion up to 0.001), "
                               "two-level grid rebuilt every frame, 1920x1080 primary + 4 area-light shadow rays/hit "
                               "+ shading; rebuild of frame N+1 on its own stream while frame N renders",
                   "l2": "inputs larger than L2 are not involved; no flush (the frames run back to back)"},
        "phase_ms": {"render": float(dyn[:, 0].mean()), "rebuild": float(dyn[:, 1].mean()), "frame": f_ms},
        "sequential": {"ms_per_frame": seq_ms, "value": rays / (seq_ms * args.steps * 1e-3) / 1e6,
                       "what": "interpolate + rebuild + render on one stream"},
        "rebuild_hidden_fraction": (seq_ms - f_ms) / max(1e-9, float(dyn[:, 1].mean())),
        "clocks": clk,
    }
    print(json.dumps(line), flush=True)


def main():
    args = parse()
    if args.impl == "reference":
        run_reference(args)
    elif args.workload == "batch":
        run_batch(args)
    elif args.workload == "serve":
        run_serve(args)
    elif args.workload == "pathtrace":
        run_pathtrace(args)
    elif args.workload == "dynamic":
        run_dynamic(args)
    else:
        run_shinobi(args)


if __name__ == "__main__":
    main()
