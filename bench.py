"""Benchmark: MC packets/s of one implicit Monte Carlo transport step on the
precision configuration (1D Type Ia-like ejecta, 256 zones, 5e5 synthetic
lines, LTE, 4096 bins, 1e7 packets; FP32 opacity tables, FP64 transport).

A step is transport::step: the per-zone opacity build (LTE solve + line
binning) followed by emission, propagation and tally normalisation of all
packets, run through the C ABI (include/sedona_gpu.h).

  value     device-resident: zone state, atomic data and tables stay in HBM;
            timed with CUDA events on the library's stream (opacity build +
            transport), L2 flushed between steps (256 MiB write).
  e2e       the same step through the C ABI with host buffers: zone state
            copied host->device (sed_set_grid), sed_step, spectrum and zone
            tallies copied device->host, wall-clock per step.
  --impl reference   the reference's own CPU implementation (built from the
            reference sources into oracle/_ref/sedona_ref) on all host cores,
            each step a bounded sample of the same workload.

Multi-GPU: packets are independent, so N ranks run N independent replicas of
the step (weak scaling); no collective is on the data path.

--workload batch64 runs the batching configuration: 64 independent 1D models
(64-512 zones, 1e5-1e7 packets each) stepped as one batch (one opacity build,
one packet launch, CUDA graphs, autotuned launch shape), against the same
models run as 64 separate plain-FP64 contexts; its reference arm runs the
reference once per model on a packet sample.

--workload adjoint runs the differentiation configuration: weighted forward +
path-replay vector-Jacobian product on the 256-zone Type Ia-like model with
absorption final, and a central-difference check of the adjoint.

--workload cart3d runs the 3D configuration instead (128^3 Cartesian cells,
1e5 lines, 2048 bins, 1e8 packets, 16 mu bins); its reference arm runs the
reference on a 32^3 grid of the same model (the reference CPU cannot hold the
128^3 x 2048 tables in host memory) and scales set_opacity by the zone count.
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

METRIC = "MC packets/s at matched spectrum chi-squared (mixed/batched vs plain FP64), 1 B200"
UNIT = "packets/s"


def captured_traffic(workload: str, n_segments: int, n_packets: int = 0):
    """DRAM bytes (read + write) of one packet-kernel launch of `workload`
    from the ncu captures in profiles/propagate_kernel_traffic.json: as
    captured where the working set stays in L2 (scale "none"), scaled from
    the captured launch by segments (scale "segments"), or a fixed part plus
    a part per packet (scale "packets": the pre-emitted state each packet
    reads).  None without a capture."""
    tfile = os.path.join(ROOT, "profiles", "propagate_kernel_traffic.json")
    if not os.path.exists(tfile):
        return None
    with open(tfile) as f:
        entries = json.load(f)
    for tr in entries if isinstance(entries, list) else [entries]:
        if tr.get("workload") != workload:
            continue
        if tr.get("scale") == "segments":
            return float(tr["dram_bytes"]) / float(tr["segments"]) * float(n_segments)
        if tr.get("scale") == "packets":
            fixed = float(tr["fixed_bytes"])
            return fixed + (float(tr["dram_bytes"]) - fixed) / float(tr["packets"]) * float(n_packets)
        return float(tr["dram_bytes"])
    return None


def captured_issue(workload: str, n_segments: int, kernel_ms: float, sm_mhz, n_sms: int):
    """Issue rate of the packet kernel: warp instructions per segment from
    the ncu capture in profiles/propagate_kernel_traffic.json
    (`warp_inst_per_segment`, `smsp__inst_executed.sum` / segments) times
    this run's segments over its kernel time, against the issue ceiling of
    one warp instruction per cycle per scheduler (4 per SM) at the SM clock
    sampled during the timed steps.  None without a capture or a clock."""
    tfile = os.path.join(ROOT, "profiles", "propagate_kernel_traffic.json")
    if not os.path.exists(tfile) or not sm_mhz or not kernel_ms:
        return None
    with open(tfile) as f:
        entries = json.load(f)
    for tr in entries if isinstance(entries, list) else [entries]:
        if tr.get("workload") != workload or "warp_inst_per_segment" not in tr:
            continue
        wps = float(tr["warp_inst_per_segment"])
        achieved = wps * float(n_segments) / (kernel_ms * 1e-3)
        peak = 4.0 * n_sms * float(sm_mhz) * 1e6
        return {"achieved": achieved, "peak": peak, "unit": "warp inst/s", "frac": achieved / peak,
                "warp_inst_per_segment": wps, "peak_basis": "4 schedulers x %d SMs x %.0f MHz (sampled)" % (n_sms, sm_mhz),
                "source": tr.get("inst_source", "profiles/propagate_kernel_traffic.json")}
    return None


def _env_rank():
    return int(os.environ.get("RANK", "0")), int(os.environ.get("WORLD_SIZE", "1")), int(os.environ.get("LOCAL_RANK", "0"))


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""

    def __init__(self, gpu: int):
        self.gpu = gpu
        self.samples = []
        self.proc = None

    def __enter__(self):
        q = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.hw_slowdown,"
             "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
             "clocks_event_reasons.sw_power_cap")
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.gpu), "--query-gpu=" + q,
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except FileNotFoundError:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            parts = [p.strip() for p in line.split(",")]
            if len(parts) >= 7:
                self.samples.append(parts)

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self) -> dict:
        if not self.samples:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["no samples"]}
        sm = [float(s[0]) for s in self.samples if s[0].replace(".", "").isdigit()]
        mx = [float(s[1]) for s in self.samples if s[1].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[k] for s in self.samples for k in range(4) if s[3 + k].lower() == "active"})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(self.samples)}


# ------------------------------------------------------------------ reference arm
def run_reference(args, workload_fn, rank: int, sample_fn=None) -> dict:
    sys.path.insert(0, os.path.join(ROOT, "oracle", "ref"))
    import run_ref
    if not run_ref.available():
        return {"impl": "reference", "unavailable": "reference harness oracle/_ref/sedona_ref is not built"}
    cores = os.cpu_count() or 1
    n_sample = args.ref_packets
    w_full = workload_fn(1)
    w = (sample_fn or workload_fn)(n_sample)
    zone_scale = w_full.zones.n_zones / w.zones.n_zones
    # warm-up (untimed), then the timed steps; each step is the reference's
    # own transport::step on a bounded packet sample
    out = run_ref.run(w, "free", threads=cores, steps=args.warmup + args.steps, timeout=3600)
    times = list(out["step_seconds"])[args.warmup:]
    t_sample = sum(times) / len(times)
    t_opac = float(out["set_opacity_seconds"][0])
    # the opacity build is per step, propagation per packet: the reference's
    # time for the full step is t_opac + (t_sample - t_opac) * N / n_sample
    # packets of a step: core packets, and decay packets when the workload has them
    frac = w.params.get("particles_n_emit_radioactive", 0) / max(int(w.params.get("core_n_emit", 1)), 1)
    n_full = int(args.packets * (1 + frac))
    n_sample_all = int(n_sample * (1 + frac))
    t = t_opac * zone_scale + max(t_sample - t_opac, 0.0) * n_full / n_sample_all
    value = n_full / t
    grid_note = "" if zone_scale == 1 else (
        " on a reduced %d-zone grid of the same model: set_opacity scaled by the zone count (x%g), "
        "propagation per packet measured on the reduced grid" % (w.zones.n_zones, zone_scale))
    # what ran is a step of n_sample_all packets (ms_per_step); the value is
    # the throughput of a full step projected from it (projected_ms_per_step)
    return {"impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": 0,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": t_sample * 1e3,
            "projected_ms_per_step": t * 1e3,
            "value_basis": "projected: %d packets / (set_opacity + propagation per packet x %d packets), "
                           "from steps of %d packets" % (n_full, n_full, n_sample_all),
            "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": w.name, "n_zones": w_full.zones.n_zones, "n_lines": w.notes.get("n_lines"),
                       "n_bins": w.nu_grid().n, "projected_packets_per_step": n_full, "threads": cores,
                       "sample_packets_per_step": n_sample_all, "sample_zones": w.zones.n_zones},
            "cpu_baseline": {"value": value, "unit": UNIT, "cores": cores, "kind": "reference",
                             "sample": "transport::step of the %s workload (%s sizes) with %d "
                                       "packets per step (%.2f s, of which set_opacity %.2f s); full-step time "
                                       "= set_opacity + propagation scaled to %d packets%s" %
                                       (w.name, "full zone/line/bin" if zone_scale == 1 else "full line/bin",
                                        n_sample_all, t_sample, t_opac, n_full, grid_note)},
            "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
            "sample_packets_per_s": n_sample_all / t_sample, "set_opacity_seconds": t_opac}


# ------------------------------------------------------------------ batches
def _timed_batch(bw, local, flush, precision, steps, warmup, tune=True, clock=False):
    """The batch stepped as one (CUDA graphs, autotuned launch shape): the
    engine, per-step stats, the tuning and the clock sampler."""
    import torch
    from pubsed_b200.batch import BatchEngine
    be = BatchEngine(bw, precision=precision, device=local, graph=True)
    # shapes timed on a quarter of every model's packets: on 2 % the short
    # trial launches are mostly tail and pick a shape ~1.5 % slower at full
    # size (128 x 7 against 256 x 4)
    tuning = be.autotune(0.25) if tune else None
    for _ in range(warmup):
        flush.fill_(1.0)
        be.step(1.0)
    stats = []
    clk = ClockSampler(local)
    with (clk if clock else _Null()):
        for i in range(steps):
            flush.fill_(float(i))
            torch.cuda.synchronize()
            stats.append(be.step(1.0))
    return be, stats, tuning, clk


def _separate(bw, local, flush, precision):
    """The batch's models as separate contexts, one after another (a warm-up
    step each, then one timed step): total device ms and the spectra."""
    import torch
    from pubsed_b200 import engine
    tot_ms, specs = 0.0, []
    for w in bw.models:
        e = engine.Engine(w, precision=precision, device=local)
        flush.fill_(1.0)
        e.step(1.0)
        flush.fill_(2.0)
        torch.cuda.synchronize()
        tot_ms += e.step(1.0)["ms_total"]
        specs.append(e.spectrum())
        e.close()
    return tot_ms, specs


def batch_leg(local, flush, packet_scale: float, steps: int = 2, warmup: int = 2) -> dict:
    """The batching configuration at `packet_scale` of its packets: batched
    mixed-precision packets/s against the same models as separate plain-FP64
    contexts, and the per-model chi^2 / dof between the two forms' spectra."""
    from pubsed_b200 import abi, workloads
    bw = workloads.batch64(packet_scale=packet_scale)
    n = bw.n_packets
    be, stats, tuning, _ = _timed_batch(bw, local, flush, abi.PREC_MIXED, steps, warmup)
    ms = sum(st["ms_total"] for st in stats) / len(stats)
    spec_b = [be.spectrum(m) for m in range(len(bw.models))]
    be.close()
    ms64, spec64 = _separate(bw, local, flush, abi.PREC_FP64)
    chi2 = [_chi2_per_dof(fb, cb, f6, c6) for (fb, cb), (f6, c6) in zip(spec_b, spec64)]
    chi2 = [c for c in chi2 if c is not None]
    return {"packet_scale": packet_scale, "packets_per_step": n, "n_models": len(bw.models),
            "mixed_batched": {"value": n / (ms * 1e-3), "ms_per_step": ms, "steps": steps, "tuning": tuning},
            "plain_fp64": {"value": n / (ms64 * 1e-3), "ms_per_step": ms64,
                           "form": "separate contexts, FP64 tables, one after another"},
            "ratio": ms64 / ms,
            "chi2_per_dof_vs_plain_fp64": {"median": float(np.median(chi2)) if chi2 else None,
                                           "max": float(np.max(chi2)) if chi2 else None, "models": len(chi2)}}


def _chi2(fa, ca, fb, cb, min_clicks=10):
    """chi^2 between two binned spectra of independent runs, sigma^2 =
    F^2 / clicks per run (equal-energy packets), over the bins with at least
    `min_clicks` packets in both: (chi^2, dof) or None."""
    use = (ca >= min_clicks) & (cb >= min_clicks)
    if not use.any():
        return None
    va = fa[use] ** 2 / ca[use]
    vb = fb[use] ** 2 / cb[use]
    return float(np.sum((fa[use] - fb[use]) ** 2 / (va + vb))), int(use.sum())


def _chi2_per_dof(fa, ca, fb, cb, min_clicks=10):
    r = _chi2(fa, ca, fb, cb, min_clicks)
    return None if r is None else r[0] / r[1]


def chi2_summary(fa, ca, fb, cb) -> dict:
    """chi^2 / dof, dof and the p-value of chi^2 for that many degrees of
    freedom (the survival function of the chi^2 distribution)."""
    from scipy import stats as sst
    r = _chi2(fa, ca, fb, cb)
    if r is None:
        return {"chi2_per_dof": None, "dof": 0, "p_value": None}
    c, dof = r
    return {"chi2_per_dof": c / dof, "dof": dof, "p_value": float(sst.chi2.sf(c, dof))}


def reference_batch(bw, n_sample: int, cores: int) -> dict:
    """The reference's own transport::step per model on `n_sample` packets
    (full zones, lines and bins); full-batch time = sum over models of
    set_opacity + propagation scaled to the model's packet count."""
    sys.path.insert(0, os.path.join(ROOT, "oracle", "ref"))
    import run_ref
    if not run_ref.available():
        return {"unavailable": "reference harness oracle/_ref/sedona_ref is not built"}
    total = t_opac_sum = 0.0
    sample_t = 0.0
    for w in bw.models:
        out = run_ref.run(w, "free", n_packets=n_sample, threads=cores, steps=1, timeout=3600)
        t_step = float(out["step_seconds"][0])
        t_opac = float(out["set_opacity_seconds"][0])
        total += t_opac + max(t_step - t_opac, 0.0) * w.n_packets / n_sample
        t_opac_sum += t_opac
        sample_t += t_step
    return {"seconds": total, "set_opacity_seconds": t_opac_sum, "sample_seconds": sample_t}


def main_batch(args, rank: int, world: int, local: int):
    """Batching configuration: 64 independent 1D models in one batch."""
    from pubsed_b200 import workloads
    bw = workloads.batch64(packet_scale=args.packet_scale)
    n_total = bw.n_packets
    cores = os.cpu_count() or 1
    n_ref = args.ref_packets or 500
    cfg = {"workload": bw.name, "n_models": len(bw.models), "zones_total": bw.n_zones,
           "n_lines": bw.notes["n_lines"], "n_bins": bw.notes["n_bins"], "packets_per_step": n_total}
    ref_sample = ("transport::step of each of the %d models with %d packets (full zones, lines, bins); batch time = "
                  "sum over models of set_opacity + propagation scaled to the model's packets" % (len(bw.models), n_ref))
    if args.impl == "reference":
        if world > 1 and rank != 0:
            return
        r = reference_batch(bw, n_ref, cores)
        if "unavailable" in r:
            print(json.dumps({"impl": "reference", "unavailable": r["unavailable"]}), flush=True)
            return
        v = n_total / r["seconds"]
        rcfg = {k: val for k, val in cfg.items() if k != "packets_per_step"}
        rcfg.update(projected_packets_per_step=n_total, sample_packets_per_model=n_ref)
        print(json.dumps({"impl": "reference", "metric": METRIC, "value": v, "unit": UNIT, "n_gpus": 0,
                          "steps": 1, "warmup": 0, "ms_per_step": r["sample_seconds"] * 1e3,
                          "projected_ms_per_step": r["seconds"] * 1e3,
                          "value_basis": "projected: per model set_opacity + propagation per packet x the "
                                         "model's packets, from steps of %d packets per model" % n_ref,
                          "higher_is_better": True,
                          "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic", "config": rcfg,
                          "cpu_baseline": {"value": v, "unit": UNIT, "cores": cores, "kind": "reference",
                                           "sample": ref_sample},
                          "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}),
              flush=True)
        return

    import torch
    from pubsed_b200 import abi
    torch.cuda.set_device(local)
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device="cuda")

    def timed_batch(precision, steps, warmup, tune=True, clock=False):
        return _timed_batch(bw, local, flush, precision, steps, warmup, tune, clock)

    be, stats, tuning, clk = timed_batch(abi.PREC_MIXED, args.steps, args.warmup, clock=True)
    ms = sum(s["ms_total"] for s in stats) / len(stats)
    kern_ms = sum(s["ms_propagate_kernel"] for s in stats) / len(stats)
    value = n_total / (ms * 1e-3)
    last = stats[-1]
    spec_b = [be.spectrum(m) for m in range(len(bw.models))]

    # end to end: every model's zone state host->device, the batched step,
    # every model's spectrum and zone tallies device->host
    e2e_t = []
    h2d = d2h = 0
    for _ in range(max(1, min(args.steps, 3))):
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        h2d = sum(be.set_zone_state(m, w.zones.rho, w.zones.T) for m, w in enumerate(bw.models))
        be.step(1.0)
        d2h = 0
        for m in range(len(bw.models)):
            f, c = be.spectrum(m)
            tal = be.tallies(m)
            d2h += f.nbytes + c.nbytes + sum(v.nbytes for v in tal.values())
        torch.cuda.synchronize()
        e2e_t.append(time.perf_counter() - t0)
    e2e = sum(e2e_t) / len(e2e_t)
    be.close()

    def separate(precision):
        return _separate(bw, local, flush, precision)

    ms64, spec64 = separate(abi.PREC_FP64)
    chi2 = [_chi2_per_dof(fb, cb, f6, c6) for (fb, cb), (f6, c6) in zip(spec_b, spec64)]
    chi2 = [c for c in chi2 if c is not None]
    out = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
           "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True, "scaling": "weak",
           "vs_baseline": None, "dtype": "f64 transport / f32 opacity tables", "data": "synthetic",
           "config": dict(cfg, precision="mixed", batched=True, segments_per_step=last["n_segments"],
                          l2="flushed between steps (256 MiB write)", tuning=tuning),
           "ms_opacity": last["ms_opacity"], "ms_transport": last["ms_transport"],
           "plain_fp64": {"value": n_total / (ms64 * 1e-3), "ms_per_step": ms64,
                          "form": "64 separate contexts, FP64 tables, one after another"},
           "chi2_per_dof_vs_plain_fp64": {"median": float(np.median(chi2)) if chi2 else None,
                                          "max": float(np.max(chi2)) if chi2 else None, "models": len(chi2)},
           "gpu_launches": int(sum(s["kernel_launches"] for s in stats)),
           "e2e": {"value": n_total / e2e, "unit": UNIT, "h2d_bytes_per_step": int(h2d),
                   "d2h_bytes_per_step": int(d2h), "ms_per_step": e2e * 1e3}}
    if not args.skip_fp64:
        ms_sm, _ = separate(abi.PREC_MIXED)
        out["separate_mixed"] = {"value": n_total / (ms_sm * 1e-3), "ms_per_step": ms_sm}
        b64, st64, _, _ = timed_batch(abi.PREC_FP64, max(1, min(args.steps, 2)), 1)
        m64 = sum(s["ms_total"] for s in st64) / len(st64)
        out["batched_fp64"] = {"value": n_total / (m64 * 1e-3), "ms_per_step": m64}
        b64.close()
    b_seg, b_pkt = 16 + 8 + 16 + 16 + 64, 264
    achieved = (last["n_segments"] * b_seg + n_total * b_pkt) / (kern_ms * 1e-3) / 1e9
    peaks = {}
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            peaks = json.load(f)
    except Exception:
        pass
    peak = float(peaks.get("hbm_gbs", 6650.0))
    out["roofline"] = {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                       "traffic": captured_traffic(bw.name, last["n_segments"]),
                       "kernel": "propagate_mixed_kernel (batched)", "kernel_ms": kern_ms,
                       "peak_source": "measured" if "hbm_gbs" in peaks else "fallback"}
    out["clocks"] = clk.summary()
    out["roofline"]["issue"] = captured_issue(bw.name, last["n_segments"], kern_ms, out["clocks"].get("sm_mhz"),
                                              torch.cuda.get_device_properties(local).multi_processor_count)
    if not args.no_cpu_baseline:
        try:
            r = reference_batch(bw, n_ref, cores)
            out["cpu_baseline"] = ({"value": None, "unit": UNIT, "cores": cores, "kind": "reference",
                                    "sample": r["unavailable"]} if "unavailable" in r else
                                   {"value": n_total / r["seconds"], "unit": UNIT, "cores": cores,
                                    "kind": "reference", "sample": ref_sample})
        except Exception as ex:  # report, do not hide
            out["cpu_baseline"] = {"value": None, "unit": UNIT, "cores": cores, "kind": "reference",
                                   "sample": "failed: %s" % str(ex)[:200]}
    print(json.dumps(out), flush=True)


# ------------------------------------------------------------------ adjoint
def main_adjoint(args, rank: int, world: int, local: int):
    """Differentiation configuration: the 256-zone Type Ia-like model with
    absorption final (radiative_eq = 0, line epsilon 1e-4), 1e7 packets,
    1024-bin spectrum, 64 frequency bands.  A step is one weighted forward
    plus the path-replay vector-Jacobian product; --fd-entries checks the
    adjoint against central differences (relative step 1e-3, common random
    numbers) on that many random (zone, band) entries."""
    from pubsed_b200 import workloads

    def wl(n):
        return workloads.type_ia(n_packets=n, epsilon=1e-4, radiative_eq=0, spectrum_bins=1024)
    n = args.packets or 10_000_000
    n_bands = 64
    cores = os.cpu_count() or 1
    cfg = {"workload": "type_ia_absorbing_adjoint", "n_zones": 256, "n_lines": 500000, "n_bins": 4096,
           "spectrum_bins": 1024, "n_bands": n_bands, "packets_per_step": n, "line_epsilon": 1e-4}
    if args.impl == "reference" or not args.no_cpu_baseline:
        ref = run_reference(argparse.Namespace(ref_packets=args.ref_packets or 20_000, warmup=1, steps=1,
                                               packets=n), wl, rank)
        if args.impl == "reference":
            if world > 1 and rank != 0:
                return
            ref["config"] = dict({k: v for k, v in cfg.items() if k != "packets_per_step"},
                                 projected_packets_per_step=n,
                                 sample_packets_per_step=ref["config"]["sample_packets_per_step"],
                                 note="reference forward only: it has no adjoint")
            print(json.dumps(ref), flush=True)
            return
    import torch
    from pubsed_b200 import abi
    from pubsed_b200.adjoint import DiffEngine
    torch.cuda.set_device(local)
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device="cuda")
    w = wl(n)
    eng = DiffEngine(w, n_bands=n_bands, precision=abi.PREC_MIXED, device=local)
    theta = np.ones((eng.nz, n_bands))
    g = np.linspace(0.5, 1.5, eng.nspec)
    clk = ClockSampler(local)
    for _ in range(args.warmup):
        flush.fill_(1.0)
        eng.forward(theta, step=0)
        eng.vjp(g)
    fw, bw, fk = [], [], []
    with clk:
        for i in range(args.steps):
            flush.fill_(float(i))
            torch.cuda.synchronize()
            _, _, st = eng.forward(theta, step=i)
            eng.vjp(g)
            fw.append(st["ms_total"])
            fk.append(st["ms_propagate_kernel"])
            bw.append(eng.last_replay["ms_total"])
    ms_f, ms_b, ms_k = (sum(x) / len(x) for x in (fw, bw, fk))
    seg = st["n_segments"]
    # end to end through the Python/C ABI with host arrays: theta in, spectrum
    # out, gradient in, theta-gradient out
    t0 = time.perf_counter()
    flux, click, _ = eng.forward(theta, step=0)
    grad = eng.vjp(g)
    e2e = time.perf_counter() - t0
    # full Jacobian once, then central differences on random entries
    eng.forward(theta, step=0)
    t0 = time.perf_counter()
    jac = eng.jacobian().reshape(eng.nspec, -1)
    ms_jac = eng.last_replay["ms_total"]
    fd = None
    if args.fd_entries > 0:
        cols = np.flatnonzero(np.abs(jac).max(axis=0) > 1e-6 * np.abs(jac).max())
        rng = np.random.default_rng(2024)
        errs = []
        flat = theta.reshape(-1)
        for q in rng.choice(cols, min(args.fd_entries, cols.size), replace=False):
            tp, tm = flat.copy(), flat.copy()
            tp[q] += 1e-3
            tm[q] -= 1e-3
            fp, _, _ = eng.forward(tp, step=0)
            fm, _, _ = eng.forward(tm, step=0)
            d = (fp - fm) / 2e-3
            a = jac[:, q]
            errs.append(float(np.linalg.norm(d - a) / np.linalg.norm(a)))
        fd = {"entries": len(errs), "relative_step": 1e-3, "common_random_numbers": True,
              "rel_err_max": max(errs), "rel_err_median": float(np.median(errs)),
              "norm": "||fd - adjoint||_2 / ||adjoint||_2 over the 1024 spectrum bins of a (zone, band) column"}
    value = n / ((ms_f + ms_b) * 1e-3)
    b_seg, b_pkt = 16 + 8 + 16 + 16 + 64, 264
    achieved = (seg * b_seg + n * b_pkt) / (ms_k * 1e-3) / 1e9
    peaks = {}
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            peaks = json.load(f)
    except Exception:
        pass
    peak = float(peaks.get("hbm_gbs", 6650.0))
    out = {"metric": METRIC + " (forward + adjoint)", "value": value, "unit": UNIT, "n_gpus": world,
           "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_f + ms_b, "higher_is_better": True,
           "scaling": "weak", "vs_baseline": None, "dtype": "f64 transport / f32 opacity tables",
           "data": "synthetic", "config": dict(cfg, segments_per_forward=seg, l2="flushed between steps (256 MiB write)"),
           "ms_forward": ms_f, "ms_adjoint_vjp": ms_b, "ms_jacobian": ms_jac,
           "escaped_fraction": float(click.sum()) / n, "fd_check": fd,
           "gpu_launches": 3 * args.steps,
           "e2e": {"value": n / e2e, "unit": UNIT, "h2d_bytes_per_step": int(theta.nbytes + g.nbytes),
                   "d2h_bytes_per_step": int(flux.nbytes + click.nbytes + grad.nbytes), "ms_per_step": e2e * 1e3},
           "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                        "traffic": None, "kernel": "propagate_kernel (weighted forward)", "kernel_ms": ms_k,
                        "peak_source": "measured" if "hbm_gbs" in peaks else "fallback"},
           "clocks": clk.summary()}
    if not args.no_cpu_baseline:
        out["cpu_baseline"] = ref.get("cpu_baseline", {"value": None, "sample": ref.get("unavailable")})
        out["cpu_baseline"]["sample"] = "reference forward (discrete absorption, no adjoint): " + \
            str(out["cpu_baseline"].get("sample"))
    print(json.dumps(out), flush=True)
    eng.close()


# ------------------------------------------------------------------ GPU arm
def main_ddmc(args, rank: int, world: int, local: int):
    """Time-dependent discrete diffusion: the reference's diffusing-pulse
    configuration (tests/diffusing_pulse/1D_ddmc) with 1e7 packets of the
    initial radiation field, every zone diffusive.  A step is one transport
    step of dt = 5e-10 s over the packets carried from the step before (the
    run advances through the warm-up steps too); value = packets carried
    through the timed steps / their device time."""
    from pubsed_b200 import workloads
    n = args.packets or 10_000_000
    n_ref = args.ref_packets or 20_000
    dt = 5e-10
    cores = os.cpu_count() or 1

    def reference_arm(n_sample, steps, warmup):
        sys.path.insert(0, os.path.join(ROOT, "oracle", "ref"))
        import run_ref
        if not run_ref.available():
            return None, "reference harness oracle/_ref/sedona_ref is not built"
        w = workloads.diffusing_pulse(n_initialize=n_sample, seed=rank)
        out = run_ref.run(w, "free", threads=cores, steps=warmup + steps, dt=dt, timeout=3600)
        times = list(out["step_seconds"])[warmup:]
        t = sum(times) / len(times)
        return n_sample / t, "transport::step of the diffusing pulse (200 zones, DDMC) with %d packets " \
            "carried per step, %d threads, %.3f s per step" % (n_sample, cores, t)

    if args.impl == "reference":
        if world > 1 and rank != 0:
            return
        v, note = reference_arm(n_ref, args.steps, args.warmup)
        if v is None:
            print(json.dumps({"impl": "reference", "unavailable": note}), flush=True)
            return
        print(json.dumps({"impl": "reference", "metric": METRIC, "value": v, "unit": UNIT, "n_gpus": 0,
                          "steps": args.steps, "warmup": args.warmup, "ms_per_step": n_ref / v * 1e3,
                          "projected_ms_per_step": n / v * 1e3,
                          "value_basis": "carried packets per second of steps of %d packets" % n_ref,
                          "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
                          "data": "synthetic", "config": {"workload": "diffusing_pulse_1d_ddmc",
                                                          "projected_packets_per_step": n, "threads": cores,
                                                          "sample_packets_per_step": n_ref},
                          "cpu_baseline": {"value": v, "unit": UNIT, "cores": cores, "kind": "reference",
                                           "sample": note},
                          "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}),
              flush=True)
        return

    import torch
    from pubsed_b200 import abi, engine
    torch.cuda.set_device(local)
    out = {}
    for prec in (abi.PREC_FP64, abi.PREC_MIXED):
        w = workloads.diffusing_pulse(n_initialize=n, seed=rank)
        eng = engine.Engine(w, precision=prec, device=local, seed_offset=rank)
        eng.initialize_particles(n, workloads.initial_e_rad(w.zones))
        for _ in range(args.warmup):
            eng.step(dt)
        torch.cuda.synchronize()
        clk = ClockSampler(local)
        stats = []
        with clk:
            for _ in range(args.steps):
                stats.append(eng.step(dt))
        torch.cuda.synchronize()
        pk = sum(int(s["n_packets"]) for s in stats)
        ms = sum(s["ms_total"] for s in stats)
        out[prec] = {"value": pk / (ms * 1e-3), "ms_per_step": ms / len(stats), "stats": stats, "clk": clk,
                     "census": eng.n_particles()}
        if prec == abi.PREC_MIXED:
            # end to end through the C ABI: zone state up, step, spectrum and
            # zone tallies down, wall clock
            e2e_pk, t0 = 0, time.perf_counter()
            h2d = d2h = 0
            for _ in range(2):
                h2d = eng.upload_grid()
                st = eng.step(dt)
                f, c = eng.spectrum()
                tal = eng.tallies()
                d2h = f.nbytes + c.nbytes + sum(v.nbytes for v in tal.values())
                e2e_pk += int(st["n_packets"])
            t_e2e = time.perf_counter() - t0
            out[prec]["e2e"] = {"value": world * e2e_pk / t_e2e, "unit": UNIT, "h2d_bytes_per_step": int(h2d),
                                "d2h_bytes_per_step": int(d2h), "ms_per_step": t_e2e / 2 * 1e3}
        eng.close()
    m = out[abi.PREC_MIXED]
    last = m["stats"][-1]
    line = {"metric": METRIC, "value": world * m["value"], "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": m["ms_per_step"], "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64 transport / f32 opacity tables", "data": "synthetic",
            "config": {"workload": "diffusing_pulse_1d_ddmc", "n_zones": 200, "packets_per_step": int(last["n_packets"]),
                       "segments_per_step": int(last["n_segments"]), "dt": dt, "precision": "mixed",
                       "l2": "tables L2-resident (200 zones x 1 bin)", "parallelism": "single"},
            "plain_fp64": {"value": out[abi.PREC_FP64]["value"], "ms_per_step": out[abi.PREC_FP64]["ms_per_step"]},
            "gpu_launches": int(sum(s["kernel_launches"] for s in m["stats"])),
            "e2e": m["e2e"], "clocks": m["clk"].summary()}
    if not args.no_cpu_baseline and rank == 0 and world == 1:
        v, note = reference_arm(n_ref, 1, 1)
        line["cpu_baseline"] = {"value": v, "unit": UNIT, "cores": cores, "kind": "reference", "sample": note}
    if rank == 0:
        print(json.dumps(line), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--workload", default="type_ia", choices=["type_ia", "cart3d", "batch64", "adjoint", "radio", "ddmc"])
    ap.add_argument("--fd-entries", type=int, default=32, help="adjoint: (zone, band) entries checked by central FD")
    ap.add_argument("--packet-scale", type=float, default=1.0, help="batch64: scales every model's packet count")
    ap.add_argument("--cells", type=int, default=128, help="cells per axis of the cart3d workload")
    ap.add_argument("--packets", type=int, default=None)
    ap.add_argument("--ref-packets", type=int, default=None)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--skip-fp64", action="store_true")
    ap.add_argument("--batch-leg-scale", type=float, default=1.0,
                    help="type_ia: packet scale of the batching leg added to the line (0: no batching leg)")
    args = ap.parse_args()
    rank, world, local = _env_rank()
    if args.workload == "batch64":
        return main_batch(args, rank, world, local)
    if args.workload == "adjoint":
        return main_adjoint(args, rank, world, local)
    if args.workload == "ddmc":
        return main_ddmc(args, rank, world, local)

    from pubsed_b200 import workloads

    sample_fn = None
    radio_frac = 0.0  # radioactive packets per core packet
    if args.workload == "radio":
        # the Type Ia step with its 56Ni/56Co decay packets: one per ten core
        # packets, the reference's Type Ia spectrum example's ratio
        # (examples/supernova/TypeIa/spectrum/param.lua: 1e5 core, 1e4 decay)
        radio_frac = 0.1

        def wl(n):
            return workloads.type_ia(n_packets=n, n_radioactive=int(n * radio_frac))
        default_packets, default_ref = 10_000_000, 20_000
    elif args.workload == "cart3d":
        def wl(n):
            return workloads.cart3d(n_packets=n, n_cells=args.cells)

        def sample_fn(n):
            return workloads.cart3d(n_packets=n, n_cells=min(32, args.cells))
        default_packets, default_ref = 100_000_000, 4000
    else:
        def wl(n):
            return workloads.type_ia(n_packets=n)
        default_packets, default_ref = 10_000_000, 20_000
    if args.packets is None:
        args.packets = default_packets
    if args.ref_packets is None:
        args.ref_packets = default_ref

    if args.impl == "reference":
        if world > 1 and rank != 0:
            return
        print(json.dumps(run_reference(args, wl, rank, sample_fn)), flush=True)
        return

    import numpy as np
    import torch
    import torch.distributed as dist
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    from pubsed_b200 import abi, engine

    torch.cuda.set_device(local)
    if world > 1:
        dist.init_process_group("nccl", timeout=__import__("datetime").timedelta(seconds=600))

    def barrier():
        if world > 1:
            dist.barrier()
        torch.cuda.synchronize()

    w = wl(args.packets)
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device="cuda")

    def run_mode(precision, steps, warmup, record_clock=False):
        eng = engine.Engine(w, precision=precision, device=local, seed_offset=rank)
        for _ in range(warmup):
            flush.fill_(1.0)
            eng.step(1.0)
        barrier()
        stats = []
        clk = ClockSampler(local)
        t0 = time.perf_counter()
        with (clk if record_clock else _Null()):
            for _ in range(steps):
                flush.fill_(float(len(stats)))
                torch.cuda.synchronize()
                stats.append(eng.step(1.0))
        barrier()
        wall = time.perf_counter() - t0
        return eng, stats, wall, clk

    # plain FP64 form (the denominator of the mixed-precision target)
    fp64 = None
    if not args.skip_fp64:
        e64, st64, wall64, _ = run_mode(abi.PREC_FP64, args.steps, min(args.warmup, 3))
        ms64 = sum(s["ms_total"] for s in st64) / len(st64)
        fp64 = {"value": int(st64[-1]["n_packets"]) / (ms64 * 1e-3), "ms_per_step": ms64}
        spec64 = e64.spectrum()
        e64.close()

    eng, stats, wall, clk = run_mode(abi.PREC_MIXED, args.steps, args.warmup, record_clock=True)
    spec32 = eng.spectrum()  # the last timed step's spectrum
    ms = [s["ms_total"] for s in stats]
    ms_step = sum(ms) / len(ms)
    # max over ranks
    t_local = torch.tensor([ms_step], dtype=torch.float64, device="cuda")
    if world > 1:
        dist.all_reduce(t_local, op=dist.ReduceOp.MAX)
    ms_max = float(t_local.item())
    n_step = int(stats[-1]["n_packets"])  # core packets (and decay packets)
    value = world * n_step / (ms_max * 1e-3)
    last = stats[-1]
    kern_ms = sum(s["ms_propagate_kernel"] for s in stats) / len(stats)

    # end-to-end through the C ABI with host buffers
    e2e_times = []
    h2d = d2h = 0
    for _ in range(max(1, min(args.steps, 3))):
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        b_in = eng.upload_grid()
        eng.step(1.0)
        flux, click = eng.spectrum()
        # the 3D J_nu array (n_zones x n_bins FP64, 34 GB at 128^3 x 2048) stays
        # on the device; its zone-scalar tallies and the spectrum come back
        tal = eng.tallies(J=(w.zones.type != abi.GRID_3D_CART))
        torch.cuda.synchronize()
        e2e_times.append(time.perf_counter() - t0)
        h2d = b_in
        d2h = flux.nbytes + click.nbytes + sum(v.nbytes for v in tal.values())
    e2e_t = sum(e2e_times) / len(e2e_times)
    t_e2e = torch.tensor([e2e_t], dtype=torch.float64, device="cuda")
    if world > 1:
        dist.all_reduce(t_e2e, op=dist.ReduceOp.MAX)
    e2e_value = world * n_step / float(t_e2e.item())

    # roofline of the packet kernel: algorithmic bytes per segment and per
    # packet (zone geometry 16 B in 1D / 24 B in 3D, {abs,scat} 8 B (FP32),
    # J RMW 16 B, e_abs RMW 16 B, force RMW 64 B per segment; 2 x 76 B state
    # + 32 B spectrum + 80 B emission CDF per packet)
    b_seg = (24 if w.zones.type == abi.GRID_3D_CART else 16) + 8 + 16 + 16 + 64
    b_pkt = 264
    alg_bytes = last["n_segments"] * b_seg + args.packets * b_pkt
    achieved = alg_bytes / (kern_ms * 1e-3) / 1e9
    peaks = {}
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            peaks = json.load(f)
    except Exception:
        pass
    peak = float(peaks.get("hbm_gbs", 6650.0))
    traffic = captured_traffic(w.name, last["n_segments"], n_step)

    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms_max, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64 transport / f32 opacity tables", "data": "synthetic",
        "config": {"workload": w.name, "n_zones": w.zones.n_zones, "n_lines": w.notes["n_lines"],
                   "n_bins": w.nu_grid().n, "packets_per_step": n_step, "precision": "mixed",
                   "radioactive_packets_per_step": int(w.params.get("particles_n_emit_radioactive", 0)),
                   "segments_per_step": last["n_segments"], "l2": "flushed between steps (256 MiB write)",
                   "parallelism": "replicas" if world > 1 else "single"},
        "ms_opacity": last["ms_opacity"], "ms_transport": last["ms_transport"],
        "plain_fp64": fp64,
        # the matched-chi^2 half of the metric: the mixed step's spectrum
        # against the plain-FP64 step's, both at the full packet count
        "chi2_vs_plain_fp64": chi2_summary(spec32[0], spec32[1], spec64[0], spec64[1]) if fp64 else None,
        "gpu_launches": int(sum(s["kernel_launches"] for s in stats)),
        "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": int(h2d), "d2h_bytes_per_step": int(d2h),
                "ms_per_step": e2e_t * 1e3},
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                     "traffic": traffic,
                     "kernel": "propagate_mixed_kernel" if w.zones.type != abi.GRID_3D_CART else "propagate_kernel",
                     "kernel_ms": kern_ms,
                     "peak_source": "measured" if "hbm_gbs" in peaks else "fallback"},
        "clocks": clk.summary(),
    }
    # what bounds the kernel: its tables stay in L2, so the HBM fraction
    # above is nominal; the issue rate against the scheduler ceiling is the
    # figure that moves with it
    line["roofline"]["issue"] = captured_issue(w.name, last["n_segments"], kern_ms, line["clocks"].get("sm_mhz"),
                                               torch.cuda.get_device_properties(local).multi_processor_count)
    if radio_frac > 0:
        # the captures are of the Type Ia step without decay packets: the
        # same kernel and tables, per-segment and per-packet figures carried over
        line["roofline"]["captured_on"] = "type_ia_1d without decay packets"
    if fp64:
        fp64["ratio_mixed_over_fp64"] = fp64["ms_per_step"] / ms_max
    eng.close()
    if args.workload == "type_ia" and args.batch_leg_scale > 0 and world == 1:
        # the batched half of the metric (64 models, by default at their full
        # packet counts)
        line["batch64"] = batch_leg(local, flush, args.batch_leg_scale)
    if not args.no_cpu_baseline and rank == 0 and world == 1:
        try:
            ref = run_reference(argparse.Namespace(ref_packets=args.ref_packets, warmup=1, steps=1,
                                                     packets=args.packets), wl, rank, sample_fn)
            if "unavailable" in ref:
                line["cpu_baseline"] = {"value": None, "unit": UNIT, "cores": os.cpu_count(), "kind": "reference",
                                        "sample": ref["unavailable"]}
            else:
                line["cpu_baseline"] = ref["cpu_baseline"]
        except Exception as ex:  # report, do not hide
            line["cpu_baseline"] = {"value": None, "unit": UNIT, "cores": os.cpu_count(), "kind": "reference",
                                    "sample": "failed: %s" % str(ex)[:200]}
    if rank == 0:
        print(json.dumps(line), flush=True)
    if world > 1:
        dist.destroy_process_group()


class _Null:
    def __enter__(self):
        return self

    def __exit__(self, *a):
        return False


if __name__ == "__main__":
    main()
