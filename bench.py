"""Benchmark of the Split transport path on the atrium workload.

Workload (one step = one cascade frame): a seeded procedural atrium of
262,144 FP32 triangles, a 1280x720 camera, screen receivers at 4x4 px
(cascade-0 spacing), 36 interval rays per receiver (about 2.1 M interval
rays per frame), 8 cascades with 32 base directions, hit shading with
emissive next-event estimation, merge of every level, probe packing, and the
world-space resolve of every pixel.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

`value` is interval rays per second of trace+merge with inputs resident in
HBM (Mrays/s, whole job over all ranks); `e2e` is the same metric through
lux_view_frame_host with host buffers, copies and the resolve included.
`--impl reference` times the CPU oracle (the restatement of the reference's
shader math) on the host cores on a bounded sample of the same workload.
"""
from __future__ import annotations

import argparse
import json
import math
import os
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "cascade trace+merge ms/frame & Mrays/s @720p: plain vs learned cache, ≤2% RMSE"
WIDTH, HEIGHT, PROBE_PX = 1280, 720, 4
TRIANGLES = 262_144
RAYS_PER_RECEIVER = 36
EYE, TARGET = (-17.0, 3.0, -15.0), (4.0, 4.0, 6.0)
L2_FLUSH_BYTES = 512 << 20
REFERENCE_SPP = 4096
# DRAM bytes per ray of the traversal kernels from one ncu capture of the
# small atrium case (65,536 triangles at 640x360: dram read + write per launch
# / rays of that launch); the full frame's traffic is scaled from it by its
# ray counts.
DRAM_BYTES_PER_INTERVAL_RAY = (4.247040e6 + 0.378880e6) / 421344
DRAM_BYTES_PER_SHADOW_RAY = (54.969600e6 + 2.205952e6) / 1237295
LEARNED_CUTOFF = 1
LEARNED_WARMUP = 200
# Kernels of one plain Split frame with world history: clear, 3 seed, the
# sample-sequence sort (radix-sort histogram, exclusive sum, 8 one-sweep passes
# over 62-bit keys, ordinal), 3 retain, layout, clear entries, closest, shade,
# shadow, deposit, the corners and history maps of every level, pack; then a
# merge per level; 4 more when visibility queries are sorted (histogram, scan
# init and scan, scatter).
LAUNCHES_PER_FRAME_FIXED = 26


def launches_per_frame(levels: int, sort_queries: bool, sort_rays: bool = False) -> int:
    """Kernels of one plain frame; sorting the interval rays adds the key
    pass to the four counting-sort launches."""
    return LAUNCHES_PER_FRAME_FIXED + levels + (4 if sort_queries else 0) + (5 if sort_rays else 0)


def settings_for_workload(sanitize: bool = True):
    """The workload's cascade settings.  sanitize=False skips liblux's
    RadianceCascades::sanitized() (the values are already in range; a test
    checks both give the same record), for the CPU arm, which loads no part
    of the library."""
    import bevy_penumbra_b200 as bp
    s = bp.RadianceCascades(probe_spacing=0.25, interval_length=0.4, levels=8, base_columns=8, base_rows=4,
                            interval_ratio=2.0, interval_rule=bp.INTERVAL_ENDS_GEOMETRIC,
                            layout=bp.LAYOUT_SPLIT, rays_per_receiver=RAYS_PER_RECEIVER, emissive_samples=16)
    return s.sanitized() if sanitize else s


def direction_count(settings, level: int) -> int:
    """Directions of a level: (base_columns x base_rows) x 4^level."""
    return (settings.base_columns * settings.base_rows) << (2 * level)


def merge_compulsory_bytes(settings, cells, history: bool) -> int:
    """Bytes the merge stage must move in one frame: per record the sample
    count and sum read (20 B) and the merged, raw and mass records written
    (40 B), with history the previous frame's raw and mass records read
    (24 B); per cell its corner ids, corner fractions and previous-frame id
    (52 B); and every level below the coarsest reads each child record once
    (16 B)."""
    total = 0
    for level in range(settings.levels):
        records = int(cells[level]) * direction_count(settings, level)
        total += records * (60 + (24 if history else 0)) + int(cells[level]) * 52
        if level + 1 < settings.levels:
            total += int(cells[level + 1]) * direction_count(settings, level + 1) * 16
    return total


def merge_roofline(settings, st, merge_ms, peak, peak_kind):
    """The merge stage (corners, history maps, merges of every level) against
    the HBM copy rate on its compulsory bytes."""
    history = settings.history_frames > 0 and (settings.temporal_blend > 0 or settings.split_transmittance_blend > 0)
    cells = list(st.cells)[:settings.levels]
    nbytes = merge_compulsory_bytes(settings, cells, history)
    achieved = nbytes / (merge_ms * 1e-3) / 1e9
    return {"kernel": ("merge stage (merge_prep_kernel: corners and history maps of every level; merge_own_kernel: the "
                       "own part of every record of every level; merge_children_kernel per level below the coarsest)"), "bound": "hbm",
            "achieved": achieved, "peak": peak, "peak_kind": peak_kind, "unit": "GB/s", "frac": achieved / peak,
            "compulsory_bytes": nbytes, "ms": merge_ms,
            "records": sum(int(c) * direction_count(settings, l) for l, c in enumerate(cells))}


def world_normals(packed, hits, dirs):
    """Geometric normals of hit triangles in world space, facing the ray."""
    sw = packed.scene_words
    gw = packed.geometry_words
    header = sw[0]
    inst = hits["instance"].astype(np.int64)
    tri = hits["triangle"].astype(np.int64)
    base = header[1] + inst * header[3]
    idx = gw[1 + tri][:, :3].astype(np.int64)
    vb = int(gw[0][1])
    verts = gw[vb + idx * 5][:, :, :3].view(np.float32).astype(np.float64)  # (n, 3, 3)
    rows = np.stack([sw[base + 3 + r].view(np.float32).astype(np.float64) for r in range(3)], axis=1)  # (n,3,4)
    world = np.einsum("nrc,nvc->nvr", rows[:, :, :3], verts) + rows[:, None, :, 3]
    n = np.cross(world[:, 1] - world[:, 0], world[:, 2] - world[:, 0])
    n /= np.maximum(np.linalg.norm(n, axis=1, keepdims=True), 1e-30)
    flip = np.sum(n * dirs, axis=1) > 0
    n[flip] = -n[flip]
    return n.astype(np.float32)


def build_workload(device: int = 0, host_only: bool = False):
    """Scene, receivers and resolve points (primary hits of the camera).

    host_only: the reference arm packs the scene with the oracle's packer and
    finds the primary hits with the CPU oracle, so it loads nothing of
    liblux (the words and hits are bit-identical either way)."""
    import bevy_penumbra_b200 as bp
    from bevy_penumbra_b200 import scenes

    t0 = time.time()
    desc = scenes.atrium(seed=2, triangles=TRIANGLES)
    if host_only:
        import oracle
        packed = oracle.OraclePacked.from_desc(desc)
        oscene = oracle.OracleScene.from_packed(packed)
    else:
        packed = bp.PackedScene.from_desc(desc)
    ctx = scene = None
    if not host_only:
        import torch
        stream = torch.cuda.current_stream(device)
        ctx = bp.LuxContext(device, stream.cuda_stream)
        scene = bp.GpuScene(ctx, packed)

    def primary(stride):
        o, d = scenes.camera_rays(WIDTH, HEIGHT, EYE, TARGET, 60.0, stride)
        rays = np.zeros(len(o), dtype=bp.RAY_DTYPE)
        rays["origin"] = o
        rays["direction"] = d
        rays["limit"] = 1e20
        if host_only:
            hits, _ = oscene.trace_rays(rays)
        else:
            import torch
            d_rays = torch.from_numpy(rays.view(np.uint8).copy()).to(f"cuda:{device}")
            d_hits = torch.zeros(len(rays) * bp.HIT_DTYPE.itemsize, dtype=torch.uint8, device=f"cuda:{device}")
            bp.trace_rays(ctx, scene, d_rays.data_ptr(), len(rays), d_hits.data_ptr())
            torch.cuda.synchronize(device)
            hits = d_hits.cpu().numpy().view(bp.HIT_DTYPE)
        ok = hits["triangle"] != 0xFFFFFFFF
        pos = np.zeros((int(ok.sum()), 4), np.float32)
        pos[:, :3] = o[ok] + d[ok] * hits["distance"][ok, None]
        nrm = np.zeros_like(pos)
        nrm[:, :3] = world_normals(packed, hits[ok], d[ok])
        # Screen attributes of the hit pixels: view depth and raster identity.
        fwd = np.asarray(TARGET, np.float64) - np.asarray(EYE, np.float64)
        fwd /= np.linalg.norm(fwd)
        screen = {"hit": ok, "depth": (hits["distance"][ok] * (d[ok] @ fwd.astype(np.float32))).astype(np.float32),
                  "identity": hits["instance"][ok].astype(np.uint32)}
        return pos, nrm, screen

    rpos, rnrm, _ = primary(PROBE_PX)
    ppos, pnrm, pscreen = primary(1)
    settings = settings_for_workload(sanitize=not host_only)
    # Exact record counts per level (cells holding a receiver x directions).
    entries = 0
    cells_max = 0
    for level in range(settings.levels):
        s = np.float32(settings.probe_spacing * (1 << level))
        cells = np.unique(np.floor(rpos[:, :3] / s).astype(np.int64), axis=0).shape[0]
        cells_max = max(cells_max, cells)
        entries += cells * direction_count(settings, level)
    view = None if host_only else bp.SplitView(ctx, max_receivers=len(rpos), max_cells=cells_max,
                                               max_entries=entries,
                                               max_rays=len(rpos) * settings.rays_per_receiver)
    if view is not None:
        # Distance LODs from the bench camera (resolve scale 1 = 1 target
        # pixel); at 1280x720 and 60 degrees the LOD-0 band reaches 156 m.
        view.set_camera(scenes.clip_from_world(EYE, TARGET, 60.0, WIDTH, HEIGHT), EYE, HEIGHT, 1)
    return dict(bp=bp, desc=desc, packed=packed, ctx=ctx, scene=scene, view=view, settings=settings, pscreen=pscreen,
                rpos=rpos,
                rnrm=rnrm, ppos=ppos, pnrm=pnrm, entries=entries, cells_max=cells_max, setup_s=time.time() - t0)


SURFACE_CLASSES = {0: "columns", 1: "arches", 2: "floor tiles", 3: "emitters", 4: "ceiling"}


def point_classes(w, indices):
    """Surface class of resolve points (the mesh of the instance each primary
    hit landed on; the atrium adds columns, arches, tiles, emitters and the
    ceiling in that order)."""
    slot = w["pscreen"]["identity"][indices].astype(np.int64)
    caller = w["packed"].instance_order.astype(np.int64)[slot]
    return np.asarray(w["desc"].instance_mesh, np.int64)[caller]


def emitter_distance(packed, points):
    """Distance (m) from each point to the nearest emissive triangle (the
    scene's emitter light records: vertex, edge1, edge2), exact in FP64: the
    plane distance where the point projects inside the triangle, else the
    nearest of its three edges."""
    rec = packed.lights[packed.conventional:].view(np.float32).astype(np.float64)
    p = np.asarray(points, np.float64)[:, :3]
    best = np.full(len(p), np.inf)
    for a, e1, e2 in zip(rec[:, 0:3], rec[:, 12:15], rec[:, 16:19]):
        n = np.cross(e1, e2)
        area2 = float(np.dot(n, n))
        if area2 <= 0.0:
            continue
        q = p - a
        # Barycentrics of the projection (solve q = u e1 + v e2 + h n).
        u = np.einsum("ij,j->i", np.cross(q, e2), n) / area2
        v = np.einsum("ij,j->i", np.cross(e1, q), n) / area2
        inside = (u >= 0) & (v >= 0) & (u + v <= 1)
        d = np.where(inside, np.abs(q @ n) / np.sqrt(area2), np.inf)
        for s0, s1 in ((a, a + e1), (a + e1, a + e2), (a + e2, a)):
            seg = s1 - s0
            t = np.clip(((p - s0) @ seg) / float(np.dot(seg, seg)), 0.0, 1.0)
            d = np.minimum(d, np.linalg.norm(p - (s0 + t[:, None] * seg), axis=1))
        best = np.minimum(best, d)
    return best


EMITTER_BANDS = (0.0, 0.25, 0.5, 1.0, 2.0, 4.0, np.inf)


def error_report(bp, ctx, est, ref, classes, distance=None):
    """lux_error_stats of an estimate against a reference, plus the relative
    RMSE and the ratio of means per surface class (host, FP64), and with the
    points' distances to the nearest emitter the same per distance band,
    with each band's share of the summed squared error."""
    out = bp.error_stats(ctx, est.data_ptr(), ref.data_ptr(), len(est))
    e, r = est.cpu().numpy().astype(np.float64), ref.cpu().numpy()
    ok = (e[:, 3] > 0) & (r[:, 3] > 0)
    per = {}
    for k, name in SURFACE_CLASSES.items():
        m = ok & (classes == k)
        if m.sum() < 8:
            continue
        d = e[m, :3] - r[m, :3]
        mean_ref = r[m, :3].mean()
        per[name] = {"points": int(m.sum()), "relative_rmse": float(np.sqrt(np.mean(d * d)) / max(mean_ref, 1e-30)),
                     "ratio_of_means": float(e[m, :3].mean() / max(mean_ref, 1e-30))}
    out["per_surface"] = per
    if distance is not None:
        m_all = ok & (classes != 3)  # emitters excluded, as in the surface classes
        sq = np.sum((e[:, :3] - r[:, :3]) ** 2, axis=1)
        total = float(sq[m_all].sum())
        bands = []
        for lo, hi in zip(EMITTER_BANDS[:-1], EMITTER_BANDS[1:]):
            m = m_all & (distance >= lo) & (distance < hi)
            if m.sum() == 0:
                continue
            mean_ref = r[m, :3].mean()
            bands.append({"from_m": lo, "to_m": None if np.isinf(hi) else hi, "points": int(m.sum()),
                          "relative_rmse": float(np.sqrt(sq[m].mean() / 3.0) / max(mean_ref, 1e-30)),
                          "ratio_of_means": float(e[m, :3].mean() / max(mean_ref, 1e-30)),
                          "share_of_squared_error": float(sq[m].sum() / max(total, 1e-300))})
        out["by_emitter_distance"] = bands
    return out


class ClockSampler:
    """SM clocks and throttle reasons sampled during the timed region: NVML
    read every 5 ms on a thread (one sample at entry and one at exit, so a
    timed region shorter than the period still has samples), or nvidia-smi
    when NVML is unavailable.  Reads settings only."""

    QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
    NAMES = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]

    def __init__(self, device: int):
        self.device = device
        self.proc = None
        self.nvml = None
        self.handle = None
        self.lines: list[str] = []
        self.samples: list[tuple] = []
        self.stop = threading.Event()
        self.thread = None

    def _nvml_handle(self):
        import pynvml
        import torch
        pynvml.nvmlInit()
        self.nvml = pynvml
        try:
            p = torch.cuda.get_device_properties(self.device)
            bus = f"{p.pci_domain_id:08x}:{p.pci_bus_id:02x}:{p.pci_device_id:02x}.0"
            return pynvml.nvmlDeviceGetHandleByPciBusId(bus)
        except Exception:
            return pynvml.nvmlDeviceGetHandleByIndex(self.device)

    def _nvml_sample(self):
        n = self.nvml
        sm = n.nvmlDeviceGetClockInfo(self.handle, n.NVML_CLOCK_SM)
        mx = n.nvmlDeviceGetMaxClockInfo(self.handle, n.NVML_CLOCK_SM)
        bits = n.nvmlDeviceGetCurrentClocksEventReasons(self.handle)
        masks = [n.nvmlClocksEventReasonHwSlowdown, n.nvmlClocksEventReasonHwThermalSlowdown,
                 n.nvmlClocksEventReasonSwThermalSlowdown, n.nvmlClocksEventReasonSwPowerCap]
        self.samples.append((float(sm), float(mx), [name for name, m in zip(self.NAMES, masks) if bits & m]))

    def _nvml_loop(self):
        while not self.stop.wait(0.005):
            try:
                self._nvml_sample()
            except Exception:
                return

    def __enter__(self):
        try:
            self.handle = self._nvml_handle()
            self._nvml_sample()
            self.thread = threading.Thread(target=self._nvml_loop, daemon=True)
            self.thread.start()
            return self
        except Exception:
            self.handle = None
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.device}", f"--query-gpu={self.QUERY}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except OSError:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *exc):
        if self.handle is not None:
            self.stop.set()
            self.thread.join(timeout=1)
            try:
                self._nvml_sample()
            except Exception:
                pass
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        sm, mx, reasons = [], [], set()
        for s, m, r in self.samples:
            sm.append(s)
            mx.append(m)
            reasons.update(r)
        for line in self.lines:
            f = [x.strip() for x in line.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx.append(float(f[2]))
            except ValueError:
                continue
            for name, val in zip(self.NAMES, f[5:9]):
                if val.lower() == "active":
                    reasons.add(name)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": [], "samples": 0}
        return {"sm_mhz": float(np.median(sm)), "sm_max_mhz": float(max(mx)), "reasons": sorted(reasons),
                "samples": len(sm), "source": "nvml" if self.samples else "nvidia-smi"}


def measured_peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(path):
        with open(path) as f:
            p = json.load(f)
        return float(p.get("hbm_gbs", 6650.0)), "measured"
    return 6650.0, "fallback"


# The CPU sample: every CPU_STRIDE-th receiver traced and merged, and every
# CPU_STRIDE-th resolve point resolved, by the oracle on all host threads
# (about 1.2 s of CPU time per sample on 16 threads).
CPU_STRIDE = 16


def cpu_sample(w, stride: int, threads: int):
    """One frame of the oracle (the CPU restatement of the reference's shader
    math) on every `stride`-th receiver, then the resolve of every
    `stride`-th resolve point from that frame's probes; timed together."""
    import oracle

    rpos = np.ascontiguousarray(w["rpos"][::stride])
    rnrm = np.ascontiguousarray(w["rnrm"][::stride])
    ppos = np.ascontiguousarray(w["ppos"][::stride])
    pnrm = np.ascontiguousarray(w["pnrm"][::stride])
    oscene = w.get("oscene") or oracle.OracleScene.from_packed(w["packed"])
    settings = w["settings"]
    t0 = time.perf_counter()
    frame = oracle.OracleFrame(oscene, settings.to_c(), rpos, rnrm, threads=threads)
    frame.resolve(ppos, pnrm)
    dt = time.perf_counter() - t0
    rays = int(frame.stats().interval_rays)
    frame.close()
    return {"rays": rays, "seconds": dt, "receivers": len(rpos), "points": len(ppos)}


def cpu_sample_text(sample, w, stride):
    full_rays = len(w["rpos"]) * RAYS_PER_RECEIVER
    return (f"every {stride}th receiver ({sample['receivers']} receivers, {sample['rays']} of {full_rays} "
            f"interval rays) traced and merged, and every {stride}th resolve point ({sample['points']} of "
            f"{len(w['ppos'])}) resolved, per step; ms_per_step is the measured sample time")


def run_reference(args, rank, world):
    """--impl reference: the CPU restatement on the host cores.  Loads no
    part of liblux: the oracle packs the scene, finds the primary hits and
    runs every frame."""
    if rank != 0:
        return
    import oracle

    w = build_workload(0, host_only=True)
    w["oscene"] = oracle.OracleScene.from_packed(w["packed"])
    threads = os.cpu_count() or 1
    for _ in range(max(args.warmup, 0)):
        cpu_sample(w, CPU_STRIDE, threads)
    times, sample = [], None
    for _ in range(args.steps):
        sample = cpu_sample(w, CPU_STRIDE, threads)
        times.append(sample["seconds"])
    dt = float(np.sum(times)) / max(args.steps, 1)
    mrays = sample["rays"] / dt / 1e6
    line = {
        "impl": "reference", "metric": METRIC, "value": mrays, "unit": "Mrays/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": dt * 1e3,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": workload_config(w),
        "cpu_baseline": {"value": mrays, "unit": "Mrays/s", "cores": threads, "kind": "port",
                         "sample": cpu_sample_text(sample, w, CPU_STRIDE)},
        "e2e": {"value": mrays, "unit": "Mrays/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def workload_config(w):
    s = w["settings"]
    return {"workload": f"atrium {TRIANGLES} tris, {WIDTH}x{HEIGHT} screen receivers at 4x4 px, 8 cascades",
            "triangles": w["desc"].world_triangles(), "receivers": int(len(w["rpos"])),
            "rays_per_receiver": RAYS_PER_RECEIVER, "interval_rays": int(len(w["rpos"]) * RAYS_PER_RECEIVER),
            "levels": s.levels, "base_directions": s.base_columns * s.base_rows,
            "emissive_samples": s.emissive_samples, "resolve_points": int(len(w["ppos"])),
            "records": int(w["entries"]), "l2": f"flushed ({L2_FLUSH_BYTES >> 20} MiB write) between steps"}


def run_learned(w, args, stream, flush, d_rpos, d_rnrm, d_ppos, d_pnrm, d_out, sub, s_ref, classes, plain_ms,
                plain_error, interval_rays, device, cutoff):
    """The learned-cache form of the same frame: levels from the cutoff on
    answered by the hash-grid MLP cache (trained online inside each frame),
    1/16 of the cascade-0 cells validated per frame with per-cell fallback.
    The cache warms up for LEARNED_WARMUP untimed frames first."""
    import torch

    bp, ctx, scene, settings = w["bp"], w["ctx"], w["scene"], w["settings"]
    n_recv, n_pts = len(w["rpos"]), len(w["ppos"])
    lview = bp.SplitView(ctx, max_receivers=n_recv, max_cells=int(w["cells_max"]),
                         max_entries=int(w["entries"]), max_rays=n_recv * settings.rays_per_receiver)
    cache = bp.LearnedCache(ctx)
    lo = w["rpos"][:, :3].min(0) - 1.0
    hi = w["rpos"][:, :3].max(0) + 1.0
    cache.set_bounds(lo, hi)
    lview.set_cache(cache, cutoff_level=cutoff, validate_period=16, error_bound=args.cache_bound,
                    train_samples=65536,
                    fallback_frames=16)
    lview.set_timing(True)

    def frame(step):
        settings.frame_index = step
        lview.trace_merge(scene, settings, d_rpos.data_ptr(), d_rnrm.data_ptr(), n_recv)

    for step in range(LEARNED_WARMUP):
        frame(step)
    torch.cuda.synchronize(device)
    ms, stages = [], []
    for step in range(args.steps):
        flush.fill_(float(step))
        start, end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        start.record(stream)
        frame(LEARNED_WARMUP + step)
        end.record(stream)
        torch.cuda.synchronize(device)
        ms.append(start.elapsed_time(end))
        t = lview.timings()
        stages.append((t.seed_ms, t.trace_ms, t.merge_ms, t.pack_ms))
    learned_ms = float(np.sum(ms)) / args.steps
    stage_ms = np.median(np.array(stages), axis=0)
    cs = lview.cache_stats()
    st = lview.stats()
    if st.error_flags or cache.stats().error_flags:
        raise RuntimeError("learned-cache frame reported an error")
    lview.resolve(settings, d_ppos.data_ptr(), d_pnrm.data_ptr(), n_pts, d_out.data_ptr())
    s_est = d_out[sub].contiguous()
    err = error_report(bp, ctx, s_est, s_ref, classes, w.get("error_distance"))
    return {
        "ms_per_step": learned_ms, "value": interval_rays / (learned_ms * 1e-3) / 1e6, "unit": "Mrays/s",
        "speedup_vs_plain": plain_ms / learned_ms,
        "stages_ms": {"seed": float(stage_ms[0]), "trace_with_cache": float(stage_ms[1]),
                      "merge": float(stage_ms[2]), "pack": float(stage_ms[3])},
        "relative_rmse": err["relative_rmse"], "plain_relative_rmse": plain_error["relative_rmse"],
        "rmse_change": err["relative_rmse"] / plain_error["relative_rmse"] - 1.0,
        "per_surface": err["per_surface"], "by_emitter_distance": err.get("by_emitter_distance"),
        "rays": {"cached": int(cs.cached_rays), "fallback": int(cs.fallback_rays),
                 "validated": int(cs.validated_rays), "trained_samples": int(cs.trained_samples),
                 "failed_cells": int(cs.failed_cells), "validated_cells": int(cs.validated_cells),
                 "validated_bias": float(cs.validated_bias)},
        "cache": {"levels": 16, "table": "2^19 x 2 BF16 per level", "base_resolution": 16, "growth": 1.5,
                  "mlp": "64 -> 4 x 64 ReLU -> 3, BF16 tcgen05", "learning_rate": 1e-3, "batch": 16384,
                  "samples_per_frame": 65536, "cutoff_level": cutoff, "validate_period": 16,
                  "error_bound": args.cache_bound, "fallback_frames": 16, "warmup_frames": LEARNED_WARMUP},
    }


def run_multi_bounce(w, args, stream, flush, d_rpos, d_rnrm, plain_ms, device, d_ppos, d_pnrm, d_out, sub, ref3,
                     classes):
    """The multi-bounce form of the same frame (RadianceCascades::multi_bounce):
    the primary cache with the secondary probes' bounce light, then the
    secondary cache traced from the primary hits (spacing and intervals x4).
    Timed like the plain frame after 8 untimed frames."""
    import dataclasses
    import torch

    bp, ctx, scene = w["bp"], w["ctx"], w["scene"]
    settings = dataclasses.replace(w["settings"], multi_bounce=True)
    n_recv = len(w["rpos"])
    mview = bp.SplitView(ctx, max_receivers=n_recv, max_cells=int(w["cells_max"]),
                         max_entries=int(w["entries"]), max_rays=n_recv * settings.rays_per_receiver)
    mview.set_timing(True)

    def frame(step):
        settings.frame_index = step
        mview.trace_merge(scene, settings, d_rpos.data_ptr(), d_rnrm.data_ptr(), n_recv)

    for step in range(max(args.warmup, 8)):
        frame(step)
    torch.cuda.synchronize(device)
    ms, sec_trace = [], []
    for step in range(args.steps):
        flush.fill_(float(step))
        start, end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        start.record(stream)
        frame(1000 + step)
        end.record(stream)
        torch.cuda.synchronize(device)
        ms.append(start.elapsed_time(end))
        sec_trace.append(mview.secondary().timings().trace_ms)
    st, sst = mview.stats(), mview.secondary().stats()
    if st.error_flags or sst.error_flags:
        raise RuntimeError("multi-bounce frame reported an error")
    mb_ms = float(np.sum(ms)) / args.steps
    mview.resolve(settings, d_ppos.data_ptr(), d_pnrm.data_ptr(), len(w["ppos"]), d_out.data_ptr())
    err3 = error_report(bp, ctx, d_out[sub].contiguous(), ref3, classes, w.get("error_distance"))
    return {"ms_per_step": mb_ms, "overhead_vs_plain": mb_ms / plain_ms,
            "error_vs_fp64_3_bounces": err3,
            "secondary_trace_ms": float(np.median(sec_trace)),
            "primary_rays": int(st.interval_rays), "secondary_rays": int(sst.interval_rays),
            "secondary_shadow_rays": int(sst.shadow_rays), "secondary_cells_level0": int(sst.cells[0]),
            "secondary": "spacing and intervals x4, receivers = the primary hits of ray frame % R"}


def run_screen(w, args, stream, flush, d_ppos, d_pnrm, d_out, device):
    """Screen reconstruction of the resolved frame at WIDTH x HEIGHT (the
    reference's temporal pass and 3 a-trous passes): the resolve output and
    the hit pixels' attributes scattered into full-screen images, then
    lux_screen_filter timed per frame with a static camera."""
    import torch

    bp, ctx, settings = w["bp"], w["ctx"], w["settings"]
    sc = w["pscreen"]
    dev = f"cuda:{device}"
    n = WIDTH * HEIGHT
    idx = torch.from_numpy(np.flatnonzero(sc["hit"])).to(dev)
    irr = torch.zeros((n, 4), dtype=torch.float32, device=dev)
    pos = torch.zeros((n, 4), dtype=torch.float32, device=dev)
    nrm = torch.zeros((n, 4), dtype=torch.float32, device=dev)
    ident = torch.zeros((n, 2), dtype=torch.int32, device=dev)
    irr[idx] = d_out
    pos[idx] = d_ppos
    pos[idx, 3] = torch.from_numpy(sc["depth"]).to(dev)
    nrm[idx] = d_pnrm
    ident[idx, 0] = torch.from_numpy(sc["identity"].view(np.int32)).to(dev)
    out = torch.zeros((n, 4), dtype=torch.float32, device=dev)
    from bevy_penumbra_b200 import scenes
    clip = scenes.clip_from_world(EYE, TARGET, 60.0, WIDTH, HEIGHT)
    screen = bp.ScreenFilter(ctx, WIDTH, HEIGHT)
    torch.cuda.synchronize(device)

    def frame():
        screen.filter(settings, irr.data_ptr(), pos.data_ptr(), nrm.data_ptr(), ident.data_ptr(), clip,
                      out.data_ptr(), spatial_filter_steps=3)

    for _ in range(max(args.warmup, 3)):
        frame()
    torch.cuda.synchronize(device)
    ms = []
    for step in range(args.steps):
        flush.fill_(float(step))
        start, end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        start.record(stream)
        frame()
        end.record(stream)
        torch.cuda.synchronize(device)
        ms.append(start.elapsed_time(end))
    _, meta = screen.read_history()
    t = float(np.median(ms))
    # Compulsory bytes per frame: temporal reads the frame inputs (irradiance,
    # position, normal 16 B, identity 8 B) and the history (72 B) and writes
    # the history; each a-trous pass reads irradiance + mask (20 B), position,
    # temporal metadata, normal and identity (56 B) and writes 20 B.
    alg = n * ((56 + 72 + 72) + 3 * (76 + 20))
    return {"ms_per_step": t, "pixels": n, "passes": "temporal + 3 a-trous (strides 1, 2, 4)",
            "achieved_gbs": alg / (t * 1e-3) / 1e9, "algorithmic_bytes": alg,
            "history_length_mean": float(meta[..., 0][meta[..., 3] > 0].mean())}


def max_over_ranks(value, dist, device):
    """Replicas: the job's time is the slowest rank's (a MAX all-reduce;
    the identity without a process group)."""
    if not dist:
        return value
    import torch
    t = torch.tensor([value], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def job_mrays(world, rays_per_rank, steps, total_ms):
    """Whole-job throughput: every rank traces its own replica of the frame."""
    return world * rays_per_rank * steps / (total_ms * 1e-3) / 1e6


def run_ours(args, rank, world):
    import torch

    device = int(os.environ.get("LOCAL_RANK", 0))
    torch.cuda.set_device(device)
    # A real stream (not the legacy default) so the library orders its work on
    # the same stream the CUDA events are recorded on.
    work_stream = torch.cuda.Stream(device)
    torch.cuda.set_stream(work_stream)
    dist = None
    if world > 1:
        import datetime

        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    w = build_workload(device)
    bp, ctx, scene, view, settings = w["bp"], w["ctx"], w["scene"], w["view"], w["settings"]
    stream = torch.cuda.current_stream(device)
    dev = f"cuda:{device}"
    d_rpos = torch.from_numpy(w["rpos"]).to(dev)
    d_rnrm = torch.from_numpy(w["rnrm"]).to(dev)
    d_ppos = torch.from_numpy(w["ppos"]).to(dev)
    d_pnrm = torch.from_numpy(w["pnrm"]).to(dev)
    d_out = torch.empty((len(w["ppos"]), 4), dtype=torch.float32, device=dev)
    flush = torch.empty(L2_FLUSH_BYTES // 4, dtype=torch.float32, device=dev)
    n_recv, n_pts = len(w["rpos"]), len(w["ppos"])
    view.set_timing(True)

    def frame(step):
        s = settings
        s.frame_index = step
        view.trace_merge(scene, s, d_rpos.data_ptr(), d_rnrm.data_ptr(), n_recv)

    from bevy_penumbra_b200.autotune import autotune
    tuned = autotune(view, lambda: frame(0))
    for step in range(args.warmup):
        frame(step)
        view.resolve(settings, d_ppos.data_ptr(), d_pnrm.data_ptr(), n_pts, d_out.data_ptr())
    torch.cuda.synchronize(device)
    st = view.stats()
    if st.error_flags:
        raise RuntimeError(f"view capacity exceeded: flags {st.error_flags}")
    interval_rays = int(st.interval_rays)
    if dist:
        dist.barrier()
    torch.cuda.synchronize(device)
    step_ms, trace_ms, merge_ms, seed_ms, pack_ms, resolve_ms = [], [], [], [], [], []
    with ClockSampler(device) as clocks:
        for step in range(args.steps):
            flush.fill_(float(step))
            start, end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            start.record(stream)
            frame(args.warmup + step)
            end.record(stream)
            torch.cuda.synchronize(device)
            step_ms.append(start.elapsed_time(end))
            t = view.timings()
            trace_ms.append(t.trace_ms)
            merge_ms.append(t.merge_ms)
            seed_ms.append(t.seed_ms)
            pack_ms.append(t.pack_ms)
            view.resolve(settings, d_ppos.data_ptr(), d_pnrm.data_ptr(), n_pts, d_out.data_ptr())
            resolve_ms.append(view.timings().resolve_ms)
    torch.cuda.synchronize(device)
    st = view.stats()
    total_ms = max_over_ranks(float(np.sum(step_ms)), dist, dev)
    ms_per_step = total_ms / args.steps
    value = job_mrays(world, interval_rays, args.steps, total_ms)

    # e2e: host buffers through lux_view_frame_host (copies + trace/merge + resolve).
    pin = lambda a: torch.from_numpy(a).pin_memory().numpy()
    h_rpos, h_rnrm, h_ppos, h_pnrm = pin(w["rpos"]), pin(w["rnrm"]), pin(w["ppos"]), pin(w["pnrm"])
    h_out = torch.empty((n_pts, 4), dtype=torch.float32).pin_memory().numpy()
    e2e_ms = []
    for step in range(args.warmup + args.steps):
        flush.fill_(float(step))
        torch.cuda.synchronize(device)
        settings.frame_index = step
        t0 = time.perf_counter()
        view.frame_host(scene, settings, h_rpos, h_rnrm, h_ppos, h_pnrm, h_out)
        dt = (time.perf_counter() - t0) * 1e3
        if step >= args.warmup:
            e2e_ms.append(dt)
    e2e_total = max_over_ranks(float(np.sum(e2e_ms)), dist, dev)
    e2e_value = job_mrays(world, interval_rays, args.steps, e2e_total)

    # FP32 error of the resolved irradiance against the FP64 path-traced
    # reference on every 97th resolve point (not timed): two diffuse vertices
    # (direct light + one bounce, the transport the cascades carry) and three
    # (the reference path tracer's default depth).
    view.resolve(settings, d_ppos.data_ptr(), d_pnrm.data_ptr(), n_pts, d_out.data_ptr())
    sub = torch.arange(0, n_pts, 97, device=dev)
    s_pos, s_nrm, s_est = d_ppos[sub].contiguous(), d_pnrm[sub].contiguous(), d_out[sub].contiguous()
    refs = {}
    for bounces in (2, 3):
        r = torch.zeros((len(sub), 4), dtype=torch.float64, device=dev)
        torch.cuda.synchronize(device)
        t0 = time.perf_counter()
        bp.path_reference(ctx, scene, settings, s_pos.data_ptr(), s_nrm.data_ptr(), len(sub), REFERENCE_SPP,
                          bounces, 99, r.data_ptr())
        refs[bounces] = (r, time.perf_counter() - t0)
    s_ref = refs[2][0]
    classes = point_classes(w, sub.cpu().numpy())
    distance = emitter_distance(w["packed"], s_pos.cpu().numpy())
    w["error_distance"] = distance
    error = error_report(bp, ctx, s_est, s_ref, classes, distance)
    error.update({"spp": REFERENCE_SPP, "bounces": 2, "sample": f"every 97th resolve point ({len(sub)})",
                  "reference_s": refs[2][1],
                  "oracle": "path-traced reference (emissive NEE + MIS, FP32 rays, FP64 sums), 2 diffuse vertices"})
    error3 = error_report(bp, ctx, s_est, refs[3][0], classes, distance)
    error3.update({"spp": REFERENCE_SPP, "bounces": 3, "reference_s": refs[3][1]})

    learned = run_learned(w, args, stream, flush, d_rpos, d_rnrm, d_ppos, d_pnrm, d_out, sub, s_ref, classes,
                          ms_per_step, error, interval_rays, device, args.cache_cutoff)
    # The operating point of the learned-cache configuration as stated:
    # cascades from level 3 on answered by the cache.
    learned3 = run_learned(w, args, stream, flush, d_rpos, d_rnrm, d_ppos, d_pnrm, d_out, sub, s_ref, classes,
                           ms_per_step, error, interval_rays, device, 3)
    multi_bounce = run_multi_bounce(w, args, stream, flush, d_rpos, d_rnrm, ms_per_step, device, d_ppos, d_pnrm,
                                    d_out, sub, refs[3][0], classes)
    view.resolve(settings, d_ppos.data_ptr(), d_pnrm.data_ptr(), n_pts, d_out.data_ptr())
    screen = run_screen(w, args, stream, flush, d_ppos, d_pnrm, d_out, device)

    # The batched and full-form workloads, summarised in the same line (one
    # GPU runs); each reports its own error instead of failing the line.
    extras = {}
    if world == 1 and not args.no_extras and not args.small:
        for key, fn in (("batched", lambda: batched_line(args, world, device)),
                        ("full", lambda: full_line(args, world, device, args.full_frames))):
            try:
                extras[key] = fn()
            except Exception as exc:  # reported, not hidden: the line carries the failure
                extras[key] = {"error": f"{type(exc).__name__}: {exc}"}
            torch.cuda.synchronize(device)

    if rank == 0:
        peak, peak_kind = measured_peaks()
        lay = scene.layout()
        alg_bytes = (int(st.nodes_visited) * lay["node_bytes"] + int(st.triangles_tested) * lay["triangle_bytes"]
                     + int(st.instances_visited) * 64)
        trace_s = float(np.median(trace_ms)) * 1e-3
        achieved = alg_bytes / trace_s / 1e9
        # The traversal's scene stays in L2: its bytes are also set against the
        # device's L2 read rate (32 MiB read 256 times in one launch) and the
        # HBM read rate of the same launch over 2 GiB, both measured here.
        l2_gbs = bp.measure_read_rate(ctx, 32 << 20, 256)
        hbm_read_gbs = bp.measure_read_rate(ctx, 2 << 30, 4)
        cpu = cpu_sample(w, CPU_STRIDE, os.cpu_count() or 1)
        line = {
            "metric": METRIC, "value": value, "unit": "Mrays/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms_per_step, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32", "data": "synthetic", "config": workload_config(w),
            "stages_ms": {"seed": float(np.median(seed_ms)), "trace": float(np.median(trace_ms)),
                          "merge": float(np.median(merge_ms)), "pack": float(np.median(pack_ms)),
                          "resolve": float(np.median(resolve_ms))},
            "rays": {"interval": interval_rays, "shadow": int(st.shadow_rays),
                     "per_interval_ray": {
                         "nodes": (int(st.nodes_visited) - int(st.shadow_nodes)) / interval_rays,
                         "triangles": (int(st.triangles_tested) - int(st.shadow_triangles)) / interval_rays,
                         "instances": (int(st.instances_visited) - int(st.shadow_instances)) / interval_rays},
                     "per_shadow_ray": {
                         "nodes": int(st.shadow_nodes) / max(int(st.shadow_rays), 1),
                         "triangles": int(st.shadow_triangles) / max(int(st.shadow_rays), 1),
                         "instances": int(st.shadow_instances) / max(int(st.shadow_rays), 1)},
                     "trace_mrays_s": interval_rays / trace_s / 1e6,
                     "all_rays_trace_mrays_s": (interval_rays + int(st.shadow_rays)) / trace_s / 1e6},
            "roofline": {"kernel": "trace stage (closest_split_kernel, shade, shadow_kernel, deposit)", "bound": "hbm",
                         "achieved": achieved, "peak": peak, "peak_kind": peak_kind, "unit": "GB/s",
                         "frac": achieved / peak,
                         "traffic": DRAM_BYTES_PER_INTERVAL_RAY * interval_rays
                         + DRAM_BYTES_PER_SHADOW_RAY * int(st.shadow_rays),
                         "traffic_note": "ncu dram bytes of the traversal kernels per frame, scaled by rays from "
                                         "the 65,536-triangle capture; the scene stays in L2",
                         "algorithmic_bytes": alg_bytes},
            "roofline_l2": {"kernel": "trace stage (closest_split_kernel, shade, shadow_kernel, deposit)",
                            "bound": "l2", "achieved": achieved, "peak": l2_gbs, "peak_kind": "measured in this run",
                            "unit": "GB/s", "frac": achieved / l2_gbs, "hbm_read_gbs": hbm_read_gbs,
                            "probe": "lux_measure_read_rate: 16-byte L1-bypassing loads, 32 MiB x 256 passes "
                                     "(L2) and 2 GiB x 4 passes (HBM), shortest of five launches"},
            "merge_roofline": merge_roofline(settings, st, float(np.median(merge_ms)), peak, peak_kind),
            "cpu_baseline": {"value": cpu["rays"] / cpu["seconds"] / 1e6, "unit": "Mrays/s",
                             "cores": os.cpu_count(), "kind": "port",
                             "sample": cpu_sample_text(cpu, w, CPU_STRIDE)},
            "e2e": {"value": e2e_value, "unit": "Mrays/s", "ms_per_step": e2e_total / args.steps,
                    "h2d_bytes_per_step": int(w["rpos"].nbytes + w["rnrm"].nbytes + w["ppos"].nbytes + w["pnrm"].nbytes),
                    "d2h_bytes_per_step": int(n_pts * 16)},
            "error_vs_fp64": error,
            "error_vs_fp64_3_bounces": error3,
            "learned": learned,
            "learned_cutoff_3": learned3,
            "multi_bounce": multi_bounce,
            "screen_filter": screen,
            **extras,
            "gpu_launches": args.steps * launches_per_frame(settings.levels, bool(tuned["best"].get("sort_queries")),
                                                            bool(tuned["best"].get("sort_rays"))),
            "autotune": {"best": tuned["best"], "frame_ms": tuned["frame_ms"],
                         "trials": [[t, round(ms, 3)] for t, ms in tuned["trials"]]},
            "clocks": clocks.summary(),
            "setup_s": w["setup_s"],
        }
        print(json.dumps(line), flush=True)
    if dist:
        dist.barrier()
        dist.destroy_process_group()


def build_batch_workload(device: int):
    """The batched configuration: 64 seeded scenes (triangles log-uniform in
    [1k, 200k]), each seen by one camera at 320x180, 640x360 or 1280x720 with
    screen receivers at 4x4 px and the atrium's cascade settings."""
    import torch

    import bevy_penumbra_b200 as bp
    from bevy_penumbra_b200 import scenes

    t0 = time.time()
    stream = torch.cuda.current_stream(device)
    ctx = bp.LuxContext(device, stream.cuda_stream)
    settings = settings_for_workload()
    dev = f"cuda:{device}"
    jobs, tris, res_counts = [], 0, {}
    for seed, triangles, (width, height) in scenes.batch_workload(seed=3, scenes=64):
        desc = scenes.batch_scene(seed, triangles)
        packed = bp.PackedScene.from_desc(desc)
        scene = bp.GpuScene(ctx, packed)
        size = 6.0 + 18.0 * np.log(triangles / 1000.0 + 1.0) / np.log(201.0)
        room_h = 3.0 + 0.25 * size
        eye = (0.05 * size, 0.45 * room_h, -0.45 * size)
        target = (-0.05 * size, 0.2 * room_h, 0.3 * size)
        o, d = scenes.camera_rays(width, height, eye, target, 60.0, PROBE_PX)
        rays = np.zeros(len(o), dtype=bp.RAY_DTYPE)
        rays["origin"], rays["direction"], rays["limit"] = o, d, 1e20
        d_rays = torch.from_numpy(rays.view(np.uint8).copy()).to(dev)
        d_hits = torch.zeros(len(rays) * bp.HIT_DTYPE.itemsize, dtype=torch.uint8, device=dev)
        torch.cuda.synchronize(device)
        bp.trace_rays(ctx, scene, d_rays.data_ptr(), len(rays), d_hits.data_ptr())
        hits = d_hits.cpu().numpy().view(bp.HIT_DTYPE)
        ok = hits["triangle"] != 0xFFFFFFFF
        pos = np.zeros((int(ok.sum()), 4), np.float32)
        pos[:, :3] = o[ok] + d[ok] * hits["distance"][ok, None]
        nrm = np.zeros_like(pos)
        nrm[:, :3] = world_normals(packed, hits[ok], d[ok])
        entries, cells_max = 0, 1
        for level in range(settings.levels):
            sp = np.float32(settings.probe_spacing * (1 << level))
            cells = np.unique(np.floor(pos[:, :3] / sp).astype(np.int64), axis=0).shape[0] if len(pos) else 0
            cells_max = max(cells_max, cells)
            entries += cells * settings.direction_count(level)
        n = len(pos)
        view = bp.SplitView(ctx, max_receivers=max(n, 1), max_cells=cells_max, max_entries=max(entries, 1),
                            max_rays=max(n, 1) * settings.rays_per_receiver)
        jobs.append(dict(scene=scene, view=view, pos=torch.from_numpy(pos).to(dev), nrm=torch.from_numpy(nrm).to(dev),
                         n=n, triangles=triangles, res=(width, height)))
        tris += triangles
        res_counts[f"{width}x{height}"] = res_counts.get(f"{width}x{height}", 0) + 1
    torch.cuda.synchronize(device)
    return dict(bp=bp, ctx=ctx, settings=settings, jobs=jobs, triangles=tris, resolutions=res_counts,
                setup_s=time.time() - t0)


def run_batched(args, rank, world):
    """--workload batched: 64 scenes per step through lux_batch_trace_merge
    (one persistent launch per trace stage, the frame replayed as a CUDA
    graph), beside the same views traced one lux_view_trace_merge at a time."""
    import torch

    device = int(os.environ.get("LOCAL_RANK", 0))
    torch.cuda.set_device(device)
    work_stream = torch.cuda.Stream(device)
    torch.cuda.set_stream(work_stream)
    line = batched_line(args, world, device)
    if rank == 0:
        print(json.dumps(line), flush=True)


def batched_line(args, world, device):
    """The batched workload's measurement (a bench line's fields)."""
    import torch

    w = build_batch_workload(device)
    bp, ctx, settings, jobs = w["bp"], w["ctx"], w["settings"], w["jobs"]
    stream = torch.cuda.current_stream(device)
    flush = torch.empty(L2_FLUSH_BYTES // 4, dtype=torch.float32, device=f"cuda:{device}")
    batch = bp.Batch(ctx)
    args_jobs = [(j["view"], j["scene"], j["pos"].data_ptr(), j["nrm"].data_ptr(), j["n"]) for j in jobs]

    def batched(step):
        settings.frame_index = step
        batch.trace_merge(args_jobs, settings)

    def one_by_one(step):
        settings.frame_index = step
        for j in jobs:
            j["view"].trace_merge(j["scene"], settings, j["pos"].data_ptr(), j["nrm"].data_ptr(), j["n"])

    # Batch launch shape: blocks per SM, the trace stage fused into one
    # cooperative launch or not, and the work-queue tile (each point: one
    # untimed frame, then one timed).
    trials = []
    for bps in (8, 16, 32):
        for fused in (0, 1):
            for tile in (32, 128):
                batch.set_tuning(bps, bps, fused, tile)
                batched(0)
                start, end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                start.record(stream)
                batched(1)
                end.record(stream)
                torch.cuda.synchronize(device)
                trials.append(((bps, fused, tile), start.elapsed_time(end)))
    best = min(trials, key=lambda t: t[1])[0]
    batch.set_tuning(best[0], best[0], best[1], best[2])

    def timed(fn):
        for step in range(args.warmup):
            fn(step)
        torch.cuda.synchronize(device)
        ms = []
        for step in range(args.steps):
            flush.fill_(float(step))
            start, end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            start.record(stream)
            fn(args.warmup + step)
            end.record(stream)
            torch.cuda.synchronize(device)
            ms.append(start.elapsed_time(end))
        return float(np.sum(ms)) / args.steps

    with ClockSampler(device) as clocks:
        batch_ms = timed(batched)
    sequential_ms = timed(one_by_one)
    rays = sum(j["n"] for j in jobs) * settings.rays_per_receiver
    info = batch.info()
    if True:
        line = {
            "metric": METRIC, "value": world * rays / (batch_ms * 1e-3) / 1e6, "unit": "Mrays/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": batch_ms, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": {"workload": "batched: 64 seeded scenes, triangles log-uniform in [1k, 200k], views from "
                                   "{320x180, 640x360, 1280x720}, receivers at 4x4 px, 8 cascades",
                       "scenes": len(jobs), "triangles": w["triangles"], "resolutions": w["resolutions"],
                       "interval_rays": rays, "rays_per_receiver": settings.rays_per_receiver,
                       "l2": f"flushed ({L2_FLUSH_BYTES >> 20} MiB write) between steps"},
            "batch": {"graph_captures": info.graph_captures, "graph_launches": int(info.graph_launches),
                      "kernels_per_frame": info.kernels_per_frame,
                      "tuning": {"blocks_per_sm": best[0], "fused_trace": best[1], "tile_rays": best[2]},
                      "tuning_trials_ms": [[list(b), round(t, 3)] for b, t in trials]},
            "sequential_views": {"ms_per_step": sequential_ms, "value": rays / (sequential_ms * 1e-3) / 1e6},
            "gpu_launches": args.steps * info.kernels_per_frame,
            "clocks": clocks.summary(), "setup_s": w["setup_s"],
        }
    batch.close()
    return line


FULL_VIEWS = [((-17.0, 3.0, -15.0), (4.0, 4.0, 6.0)), ((17.0, 3.5, -15.0), (-4.0, 4.0, 6.0)),
              ((-17.0, 4.0, 15.0), (4.0, 3.0, -6.0)), ((17.0, 3.0, 15.0), (-4.0, 4.0, -6.0))]
FULL_WIDTH, FULL_HEIGHT, FULL_FPS = 1920, 1080, 60.0


def primary_receivers(bp, ctx, scene, packed, eye, target, width, height, stride, device):
    """World-space primary hits (position, facing normal) through every
    stride-th pixel block of a camera (the G-buffer receivers)."""
    import torch

    from bevy_penumbra_b200 import scenes
    o, d = scenes.camera_rays(width, height, eye, target, 60.0, stride)
    rays = np.zeros(len(o), dtype=bp.RAY_DTYPE)
    rays["origin"], rays["direction"], rays["limit"] = o, d, 1e20
    dev = f"cuda:{device}"
    d_rays = torch.from_numpy(rays.view(np.uint8).copy()).to(dev)
    d_hits = torch.zeros(len(rays) * bp.HIT_DTYPE.itemsize, dtype=torch.uint8, device=dev)
    torch.cuda.synchronize(device)
    bp.trace_rays(ctx, scene, d_rays.data_ptr(), len(rays), d_hits.data_ptr())
    hits = d_hits.cpu().numpy().view(bp.HIT_DTYPE)
    ok = hits["triangle"] != 0xFFFFFFFF
    pos = np.zeros((int(ok.sum()), 4), np.float32)
    pos[:, :3] = o[ok] + d[ok] * hits["distance"][ok, None]
    nrm = np.zeros_like(pos)
    nrm[:, :3] = world_normals(packed, hits[ok], d[ok])
    return pos, nrm


def run_full(args, rank, world):
    """--workload full: a 1,048,576-triangle scene whose 4 emitters move on
    circles at 0.5 m/s (60 frames per second) and whose 8 rigid boxes move in
    turn every 30 frames, seen by 4 views at 1920x1080 (receivers at 4x4 px);
    every frame refits the TLAS with the new poses and emitter records, the
    views invalidate history around what moved, and trace+merge runs per
    view.  The plain form runs all frames, then the learned-cache form replays
    the same motion; the final frame of each is compared with a 4096-spp FP64
    reference on every 64th receiver of every view."""
    import torch

    import bevy_penumbra_b200 as bp
    from bevy_penumbra_b200 import scenes

    device = int(os.environ.get("LOCAL_RANK", 0))
    torch.cuda.set_device(device)
    work_stream = torch.cuda.Stream(device)
    torch.cuda.set_stream(work_stream)
    line = full_line(args, world, device, args.frames)
    if rank == 0:
        print(json.dumps(line), flush=True)


def full_line(args, world, device, frames):
    """The full-form workload's measurement over `frames` frames of motion."""
    import torch

    import bevy_penumbra_b200 as bp
    from bevy_penumbra_b200 import scenes

    stream = torch.cuda.current_stream(device)
    dev = f"cuda:{device}"
    t0 = time.time()
    desc, emitters, boxes = scenes.full_scene(5, 1 << 20)
    packed = bp.PackedScene.from_desc(desc)
    ctx = bp.LuxContext(device, stream.cuda_stream)
    scene = bp.GpuScene(ctx, packed)
    slot_of = np.empty(len(packed.instance_order), np.int64)
    slot_of[packed.instance_order.astype(np.int64)] = np.arange(len(packed.instance_order))
    base = np.stack([desc.instance_transform[int(i)] for i in packed.instance_order]).astype(np.float64)
    orbits = scenes.emitter_orbits(desc, emitters)
    box_rng = np.random.default_rng(55)
    box_steps = [box_rng.uniform(-0.6, 0.6, size=3) * (1.0, 0.0, 1.0) for _ in range(64)]
    settings = settings_for_workload()
    mesh_lo = {m: desc.meshes[m].positions.min(0) for m in set(desc.instance_mesh)}
    mesh_hi = {m: desc.meshes[m].positions.max(0) for m in set(desc.instance_mesh)}

    def world_box(inst, m):
        lo, hi = mesh_lo[desc.instance_mesh[inst]], mesh_hi[desc.instance_mesh[inst]]
        corners = np.array([[x, y, z] for x in (lo[0], hi[0]) for y in (lo[1], hi[1]) for z in (lo[2], hi[2])])
        w = corners @ m[:, :3].T + m[:, 3]
        return w.min(0), w.max(0)

    def poses(frame):
        """Slot-ordered poses at `frame`, and the (instance, old, new) moves."""
        cur = base.copy()
        t = frame / FULL_FPS
        for (c, r, phase, sign), inst in zip(orbits, emitters):
            a = phase + sign * 0.5 * t / r
            cur[slot_of[inst], :, 3] = c + r * np.array([math.cos(a), 0.0, math.sin(a)])
        for k in range(frame // 30):
            inst = boxes[k % len(boxes)]
            cur[slot_of[inst], :, 3] += box_steps[k % len(box_steps)]
        return cur

    stride = PROBE_PX
    # Views sized for the receivers of the first frame with headroom (moved
    # boxes change the receiver set a little).
    recv = [primary_receivers(bp, ctx, scene, packed, e, tgt, FULL_WIDTH, FULL_HEIGHT, stride, device)
            for e, tgt in FULL_VIEWS]
    views = []
    for pos, _ in recv:
        entries, cells_max = 0, 1
        for level in range(settings.levels):
            sp = np.float32(settings.probe_spacing * (1 << level))
            cells = np.unique(np.floor(pos[:, :3] / sp).astype(np.int64), axis=0).shape[0]
            cells_max = max(cells_max, int(cells * 1.25) + 64)
            entries += int(cells * 1.25 + 64) * settings.direction_count(level)
        views.append(bp.SplitView(ctx, max_receivers=int(len(pos) * 1.1), max_cells=cells_max,
                                  max_entries=entries, max_rays=int(len(pos) * 1.1) * settings.rays_per_receiver))
    setup_s = time.time() - t0

    def receivers_now():
        rec = [primary_receivers(bp, ctx, scene, packed, e, tgt, FULL_WIDTH, FULL_HEIGHT, stride, device)
               for e, tgt in FULL_VIEWS]
        out = []
        for v, (p, nm) in zip(views, rec):
            n = min(len(p), int(v.desc.max_receivers))
            out.append((torch.from_numpy(p[:n]).to(dev), torch.from_numpy(nm[:n]).to(dev), n))
        return out

    def run_form(cache):
        for v in views:
            v.reset_history()
            if cache is None:
                v.set_cache(None)
            else:
                v.set_cache(cache, cutoff_level=args.cache_cutoff, validate_period=16, error_bound=args.cache_bound,
                            train_samples=65536, fallback_frames=16)
        prev = poses(0)
        scene.refit(prev, lights=packed.lights_at(prev))
        d_rec = receivers_now()
        ms, rays = [], 0
        for frame in range(frames):
            cur = poses(frame)
            moved = [i for i in range(len(cur)) if not np.array_equal(cur[i], prev[i])]
            box_moved = any(int(packed.instance_order[sl]) in boxes for sl in moved)
            if box_moved:
                # A rigid box moved: refit, then the G-buffer (receivers) changes.
                scene.refit(cur, lights=packed.lights_at(cur))
                d_rec = receivers_now()
            start, end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            start.record(stream)
            if moved and not box_moved:
                scene.refit(cur, lights=packed.lights_at(cur))
            for slot in moved:
                inst = int(packed.instance_order[slot])
                lo0, hi0 = world_box(inst, prev[slot])
                lo1, hi1 = world_box(inst, cur[slot])
                for v in views:
                    v.invalidate_bounds(np.minimum(lo0, lo1), np.maximum(hi0, hi1))
            settings.frame_index = frame
            for v, (p, nm, n) in zip(views, d_rec):
                v.trace_merge(scene, settings, p.data_ptr(), nm.data_ptr(), n)
            end.record(stream)
            torch.cuda.synchronize(device)
            if frame >= 10:
                ms.append(start.elapsed_time(end))
            rays = sum(n for _, _, n in d_rec) * settings.rays_per_receiver
            prev = cur
        for v in views:
            if v.stats().error_flags:
                raise RuntimeError("full form: a view's capacity was exceeded")
        # FP64 reference on every 64th receiver of every view (final pose).
        errs = []
        for v, (p, nm, n) in zip(views, d_rec):
            sub = torch.arange(0, n, 64, device=dev)
            s_pos, s_nrm = p[sub].contiguous(), nm[sub].contiguous()
            out = torch.empty((len(sub), 4), dtype=torch.float32, device=dev)
            v.resolve(settings, s_pos.data_ptr(), s_nrm.data_ptr(), len(sub), out.data_ptr())
            ref = torch.zeros((len(sub), 4), dtype=torch.float64, device=dev)
            bp.reference_irradiance(ctx, scene, settings, s_pos.data_ptr(), s_nrm.data_ptr(), len(sub), 4096, 7,
                                    ref.data_ptr())
            errs.append((out, ref))
        est = torch.cat([e for e, _ in errs]).contiguous()
        ref = torch.cat([r for _, r in errs]).contiguous()
        err = bp.error_stats(ctx, est.data_ptr(), ref.data_ptr(), len(est))
        frame_ms = float(np.mean(ms))
        return {"ms_per_frame": frame_ms, "value": rays / (frame_ms * 1e-3) / 1e6, "interval_rays_per_frame": rays,
                "relative_rmse": err["relative_rmse"], "rmse": err["rmse"], "points": err["points"]}

    with ClockSampler(device) as clocks:
        plain = run_form(None)
        cache = bp.LearnedCache(ctx)
        lo = np.min([p[:, :3].min(0) for p, _ in recv], axis=0) - 1.0
        hi = np.max([p[:, :3].max(0) for p, _ in recv], axis=0) + 1.0
        cache.set_bounds(lo, hi)
        learned = run_form(cache)
    if True:
        line = {
            "metric": METRIC, "value": world * plain["value"], "unit": "Mrays/s", "n_gpus": world,
            "steps": frames, "warmup": 10, "ms_per_step": plain["ms_per_frame"], "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": {"workload": "full: 1,048,576 tris, 4 emitters on circles at 0.5 m/s, 8 rigid boxes moved in "
                                   "turn every 30 frames, 4 views at 1920x1080 (receivers at 4x4 px), 8 cascades",
                       "frames": frames, "fps": FULL_FPS, "views": len(views),
                       "interval_rays_per_frame": plain["interval_rays_per_frame"],
                       "reference": "4096-spp FP64 reference on every 64th receiver, final frame"},
            "plain": plain,
            "learned": dict(learned, speedup_vs_plain=plain["ms_per_frame"] / learned["ms_per_frame"],
                            rmse_change=learned["relative_rmse"] / plain["relative_rmse"] - 1.0,
                            cutoff_level=args.cache_cutoff, error_bound=args.cache_bound),
            "clocks": clocks.summary(), "setup_s": setup_s,
        }
    return line


def run_frames(args):
    """--frames-only: plain frames for ncu captures (a fixed launch sequence:
    8 merge launches per frame at 8 cascades)."""
    import torch

    from bevy_penumbra_b200.autotune import START, tuning_of
    torch.cuda.set_device(0)
    w = build_workload(0)
    view, scene, settings = w["view"], w["scene"], w["settings"]
    d_rpos = torch.from_numpy(w["rpos"]).cuda()
    d_rnrm = torch.from_numpy(w["rnrm"]).cuda()
    view.set_tuning(**tuning_of(START))
    view.set_timing(True)
    warm = 0
    if args.learned_frames:
        bp = w["bp"]
        cache = bp.LearnedCache(w["ctx"])
        cache.set_bounds(w["rpos"][:, :3].min(0) - 1.0, w["rpos"][:, :3].max(0) + 1.0)
        view.set_cache(cache, cutoff_level=args.cache_cutoff, validate_period=16, error_bound=args.cache_bound,
                       train_samples=65536, fallback_frames=16)
        warm = LEARNED_WARMUP
    stages = []
    for step in range(warm):
        settings.frame_index = step
        view.trace_merge(scene, settings, d_rpos.data_ptr(), d_rnrm.data_ptr(), len(w["rpos"]))
    torch.cuda.synchronize()
    torch.cuda.nvtx.range_push("frames")  # the launches a capture may select (ncu --nvtx-include frames/)
    for step in range(warm, warm + args.warmup + args.steps):
        settings.frame_index = step
        view.trace_merge(scene, settings, d_rpos.data_ptr(), d_rnrm.data_ptr(), len(w["rpos"]))
        torch.cuda.synchronize()
        t = view.timings()
        if step >= warm + args.warmup:
            stages.append((t.seed_ms, t.trace_ms, t.merge_ms, t.pack_ms))
    torch.cuda.nvtx.range_pop()
    st = view.stats()
    m = np.median(np.array(stages), axis=0)
    interval_rays = max(int(st.interval_rays), 1)
    print(json.dumps({"profile": "learned-frames" if args.learned_frames else "frames-only", "width": WIDTH, "height": HEIGHT, "triangles": TRIANGLES,
                      "tuning": tuning_of(START), "seed_ms": m[0], "trace_ms": m[1], "merge_ms": m[2], "pack_ms": m[3],
                      "per_interval_ray": {"nodes": (int(st.nodes_visited) - int(st.shadow_nodes)) / interval_rays,
                                           "triangles": (int(st.triangles_tested) - int(st.shadow_triangles)) / interval_rays},
                      "per_shadow_ray": {"nodes": int(st.shadow_nodes) / max(int(st.shadow_rays), 1),
                                         "triangles": int(st.shadow_triangles) / max(int(st.shadow_rays), 1)},
                      "cells": list(st.cells)[:settings.levels], "error_flags": int(st.error_flags)}))


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="atrium", choices=["atrium", "batched", "full"],
                    help="atrium: the headline frame; batched: 64 scenes per step through lux_batch_trace_merge; "
                         "full: moving emitters and boxes, 4 views at 1080p, plain and learned forms")
    ap.add_argument("--frames", type=int, default=600, help="full workload: frames of motion")
    ap.add_argument("--full-frames", type=int, default=120,
                    help="default line: frames of motion of its full-form summary")
    ap.add_argument("--no-extras", action="store_true",
                    help="default line without the batched and full-form summaries")
    ap.add_argument("--cache-cutoff", type=int, default=LEARNED_CUTOFF,
                    help="learned-cache form: first cascade answered by the cache")
    ap.add_argument("--cache-bound", type=float, default=8.0,
                    help="learned-cache form: relative bias above which a validated cell falls back")
    ap.add_argument("--small", action="store_true",
                    help="profiling case: 65,536-triangle atrium at 640x360 (not a benchmark line)")
    ap.add_argument("--frames-only", action="store_true",
                    help="profiling target: --warmup + --steps plain frames of the atrium workload with the "
                         "autotuner's starting tuning (no search, no other forms); prints the stage times")
    ap.add_argument("--learned-frames", action="store_true",
                    help="with --frames-only: learned-cache frames (cutoff --cache-cutoff) after the cache's "
                         "warm-up frames")
    args = ap.parse_args()
    if args.small:
        global WIDTH, HEIGHT, TRIANGLES, EYE, TARGET
        WIDTH, HEIGHT, TRIANGLES = 640, 360, 65_536
        EYE, TARGET = (-7.0, 3.0, -6.0), (2.0, 4.0, 3.0)
    rank = int(os.environ.get("RANK", 0))
    world = int(os.environ.get("WORLD_SIZE", 1))
    if args.frames_only:
        run_frames(args)
    elif args.impl == "reference":
        run_reference(args, rank, world)
    elif args.workload == "batched":
        run_batched(args, rank, world)
    elif args.workload == "full":
        run_full(args, rank, world)
    else:
        run_ours(args, rank, world)


if __name__ == "__main__":
    main()
