#!/usr/bin/env python
"""Benchmark of pconf's Hamiltonian build on one B200 (or N independent replicas).

Workload: the config-2 system (3 valence electrons, 120 relativistic orbitals
n <= 20, l <= 4, odd parity, M_J = 1/2, singles + doubles from 20 reference
configurations, seeded synthetic integrals, FP64 values).  One step = one
FormH: configuration adjacency, count pass, scan and fill pass, from the
device-resident determinant list and integral tables to the device-resident
lower-triangle CSR (NumH non-zeros).  Metric: H-build nnz/s.

  value  -- NumH / device time of FormH (CUDA events on the library stream),
            inputs resident in HBM; L2 flushed (512 MiB write) before each step.
  e2e    -- the same metric through the C ABI from pinned host arrays:
            set_basis + set_integrals (host->device) + form_h + NumH/Hmin back.
  --impl reference -- the oracle (C restatement of the reference's FormH) on
            the host cores, rows sampled per step.

Time to roots (key "time_to_roots", skipped with --no-roots): the config-3
system's 10 roots (4 valence electrons, 140 orbitals, Nd 1.3M) to residual
1e-8 against the FP64 H through the batched solver with one block, FormH +
solve each, in three forms: fp64 (FP64 SpMM, diagonal correction), mixed
(FP32 SpMM phase, then FP64 to the criterion) and learned_mixed (the mixed
form with the learned correction, trained first on the solver's own runs of
four smaller systems of the same orbital basis; skipped with --no-learned).
Each SpMM is set against HBM and against the measured L2 reduction
throughput that bounds it.

Batched form (key "batched", skipped with --no-batched): 64 synthetic ions
(seeds 1000-1063; 2-4 valence electrons, 30-120 orbitals, mixed M and
parity, 2k-400k determinants log-uniform), each H built on the device in
FP32, then 6 roots of every block to residual 1e-8 in one batch (SpMM
variant from the tuning cache ~/.cache/pci_b200/spmm_tune_cache.txt, tuned
and appended when absent); reported: H-build + solve time, iterations, SpMM roofline.

Multi-GPU: replicas only (the build of one system does not shard across GPUs
in this engine); every rank builds the same system, value = total NumH / max
time over ranks.
"""
from __future__ import annotations

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

MEASURED_PEAK_FALLBACK = 6650.0


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--config", default="cfg2")
    ap.add_argument("--cpu-rows", type=int, default=2000, help="rows per CPU sample step")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-fp32-form", action="store_true", help="skip the FP32 Davidson form")
    ap.add_argument("--no-batched", dest="batched", action="store_false", help="skip the batched form")
    ap.add_argument("--no-roots", dest="roots", action="store_false",
                    help="skip the time-to-roots solves of the configuration")
    ap.add_argument("--roots-config", default="cfg3", help="configuration of the time-to-roots section")
    ap.add_argument("--no-learned", dest="learned", action="store_false",
                    help="skip the learned form of the time-to-roots section")
    ap.add_argument("--learn-nd", type=int, default=30000,
                    help="determinants of each training system of the learned correction")
    ap.add_argument("--switch-tol", type=float, default=1e-5, help="residual that ends the FP32 phase")
    ap.add_argument("--profile-case", default=None,
                    help="only a short batched solve of this configuration, for profiler captures")
    ap.add_argument("--case-iters", type=int, default=6, help="iterations of --profile-case")
    ap.add_argument("--case-train", type=int, default=0, help="training epochs before --profile-case's solve")
    ap.add_argument("--batch-blocks", type=int, default=64)
    ap.add_argument("--batch-variant", type=int, default=-1, help="SpMM variant of the batched form "
                    "(-1: from the tuning cache, tuned when absent)")
    ap.add_argument("--tune-cache", default=None, help="SpMM tuning cache of the batched form "
                    "(default: ~/.cache/pci_b200/spmm_tune_cache.txt; empty string = tune every run)")
    ap.add_argument("--no-lsj", action="store_true", help="skip the LSJ section")
    ap.add_argument("--no-csf", action="store_true", help="skip the CSF-basis section")
    ap.add_argument("--davidson-iters", type=int, default=2,
                    help="plain FP64 Davidson iterations timed after the H-build (0 skips)")
    return ap.parse_args()


# DRAM bytes (dram__bytes_read.sum + dram__bytes_write.sum) the fill kernel
# moves per stored element, from an ncu capture of the same kernel on the mid
# system (NumH 1.64e8: 358 MB read + 1985 MB written); the full-size launch
# is too large to capture and its traffic grows with the stored elements.
FILL_DRAM_BYTES_PER_NNZ = (358.172416e6 + 1985.190e6) / 164067833


def peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        d = json.load(open(p))
        return float(d.get("hbm_gbs", MEASURED_PEAK_FALLBACK)), "measured"
    return MEASURED_PEAK_FALLBACK, "fallback"


class Clocks:
    """nvidia-smi sampling of SM clocks and throttle reasons during the timed region."""
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device):
        self.device = device
        self.f = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
        self.p = None

    def start(self):
        try:
            self.p = subprocess.Popen(["nvidia-smi", f"--id={self.device}", f"--query-gpu={self.Q}",
                                       "--format=csv,noheader,nounits", "-lms", "200"],
                                      stdout=self.f, stderr=subprocess.DEVNULL)
        except OSError:
            self.p = None

    def stop(self):
        if self.p is None:
            return None
        self.p.terminate()
        try:
            self.p.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.p.kill()
        self.f.flush()
        rows = []
        for line in open(self.f.name):
            parts = [x.strip() for x in line.split(",")]
            if len(parts) >= 9:
                rows.append(parts)
        os.unlink(self.f.name)
        if not rows:
            return None
        sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in rows for i in range(4) if r[5 + i] == "Active"})
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(rows)}


def algorithmic_bytes_fill(sysm, numh, value_bytes=8):
    """Bytes the fill pass must move: CSR out (col + value), row pointers in,
    determinant occupation lists in, the radial-integral table read once."""
    return (numh * (value_bytes + 4) + (sysm.nd + 1) * 8 + sysm.nd * sysm.ne * 2
            + sysm.ngint * 8 + sysm.hint_lut.nbytes)


def cpu_sample(sysm, nrows, seed, threads=0):
    """Oracle FormH over `nrows` random rows (count pass: every element evaluated,
    zeros dropped); returns (seconds, nnz)."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O
    o = O.Oracle(sysm)
    rng = np.random.default_rng(seed)
    rows = np.sort(rng.choice(np.arange(1, sysm.nd + 1), size=min(nrows, sysm.nd), replace=False))
    t, nnz, _ = o.form_h_timed_sample([(int(r), int(r)) for r in rows], threads=threads)
    return t, nnz, rows.size


def dist_setup(backend):
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    if ws == 1:
        return 0, 1, 0, None
    import torch.distributed as dist
    from datetime import timedelta
    os.environ.setdefault("MASTER_ADDR", "127.0.0.1")
    dist.init_process_group(backend, timeout=timedelta(seconds=600))
    return dist.get_rank(), dist.get_world_size(), int(os.environ.get("LOCAL_RANK", "0")), dist


def max_over_ranks(x, dist, device=None):
    if dist is None:
        return x
    import torch
    t = torch.tensor([x], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def run_reference(args):
    rank, world, local, dist = dist_setup("gloo")
    if rank != 0:
        if dist is not None:
            dist.destroy_process_group()
        return 0
    from pci_b200 import system as S
    sysm = S.make_system(**S.CONFIGS[args.config]())
    threads = os.cpu_count() or 1
    for w in range(args.warmup):
        cpu_sample(sysm, max(args.cpu_rows // 4, 8), 1000 + w, threads)
    tot_t = tot_n = tot_rows = 0
    for k in range(args.steps):
        t, n, r = cpu_sample(sysm, args.cpu_rows, 2000 + k, threads)
        tot_t += t
        tot_n += n
        tot_rows += r
    value = tot_n / tot_t
    line = {
        "metric": f"H-build nnz/s ({args.config})", "value": value, "unit": "nnz/s", "impl": "reference",
        "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": 1e3 * tot_t / args.steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded)",
        "config": {"workload": f"{args.config}: FormH of Nd={sysm.nd} determinants", "Nd": sysm.nd,
                   "rows_per_step": args.cpu_rows},
        "cpu_baseline": {"value": value, "unit": "nnz/s", "cores": threads, "kind": "port",
                         "sample": f"{args.cpu_rows} random rows of FormH per step (oracle restatement "
                                   f"of src/pconf.F90:1227-1290, OpenMP over rows)"},
        "e2e": {"value": value, "unit": "nnz/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)
    if dist is not None:
        dist.destroy_process_group()
    return 0


def pinned(a):
    import torch
    return torch.from_numpy(np.ascontiguousarray(a)).pin_memory().numpy()


def run_ours(args):
    import torch
    rank, world, local, dist = dist_setup("nccl")
    torch.cuda.set_device(local)
    from pci_b200 import system as S
    from pci_b200.capi import Engine
    sysm = S.make_system(**S.CONFIGS[args.config]())
    # host inputs in pinned memory (the e2e leg copies from these every step)
    for name in ("iarr", "nh", "jz", "ndc", "hint_lut", "gaunt_lut", "rint2", "iint2", "iint3"):
        setattr(sysm, name, pinned(getattr(sysm, name)))
    h2d = sum(getattr(sysm, n).nbytes for n in ("iarr", "nh", "jz", "ndc", "hint_lut", "gaunt_lut",
                                                  "rint2", "iint2", "iint3"))
    h2d += 4 * 4 * sysm.nsu
    eng = Engine(local)
    eng.load_system(sysm)
    flush = torch.empty(512 * 1024 * 1024, dtype=torch.uint8, device=f"cuda:{local}")
    for _ in range(args.warmup):
        eng.form_h(64)
    torch.cuda.synchronize()
    if dist is not None:
        dist.barrier()
    clocks = Clocks(local)
    clocks.start()
    t_dev, t_fill, t_count, t_adj, t_comp = [], [], [], [], []
    single = 0.0
    launches = 0
    numh = 0
    for _ in range(args.steps):
        flush.zero_()
        torch.cuda.synchronize()
        numh, numzero, hmin = eng.form_h(64)
        st = eng.stats()
        t_dev.append(st["formh_ms"])
        t_fill.append(st["formh_fill_ms"])
        t_count.append(st["formh_count_ms"])
        t_adj.append(st["adjacency_ms"])
        t_comp.append(st["formh_compact_ms"])
        single = st["formh_single_eval"]
        launches += int(st["formh_launches"]) + 1
    torch.cuda.synchronize()
    clk = clocks.stop()
    if dist is not None:
        dist.barrier()
    ms = float(np.mean(t_dev))
    ms_max = max_over_ranks(ms, dist, device=f"cuda:{local}")
    value = world * numh / (ms_max * 1e-3)
    # e2e through the C ABI from pinned host buffers
    e2e = None
    if not args.no_e2e:
        te = []
        for _ in range(args.steps):
            flush.zero_()
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            eng.load_system(sysm)
            n2, z2, hm2 = eng.form_h(64)
            te.append(time.perf_counter() - t0)
        e_s = max_over_ranks(float(np.mean(te)), dist, device=f"cuda:{local}")
        e2e = {"value": world * numh / e_s, "unit": "nnz/s", "h2d_bytes_per_step": int(h2d),
               "d2h_bytes_per_step": 24, "seconds_per_step": e_s}
    peak, peak_kind = peaks()
    fill_bytes = algorithmic_bytes_fill(sysm, numh)
    achieved = fill_bytes / (float(np.mean(t_fill)) * 1e-3) / 1e9
    line = {
        "metric": f"H-build nnz/s ({args.config})", "value": value, "unit": "nnz/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_max, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded)",
        "config": {"workload": f"{args.config}: FormH of Nd={sysm.nd} determinants, Ne={sysm.ne}, "
                               f"Nc={sysm.nc}, Ngint={sysm.ngint}",
                   "Nd": sysm.nd, "NumH": int(numh), "numzero": int(numzero), "Hmin": hmin,
                   "l2": "flushed (512 MiB write) before every step; CSR output 12 B x NumH >> L2",
                   "parallelism": f"replicas x{world}"},
        "breakdown_ms": {"adjacency": float(np.mean(t_adj)), "count": float(np.mean(t_count)),
                         "fill": float(np.mean(t_fill)), "compact": float(np.mean(t_comp))},
        "formh_build": "single evaluation (candidate bound, padded fill, compaction)" if single
                       else "two passes (count, fill)",
        "roofline": {"bound": "hbm", "kernel": "k_tiles fill pass", "achieved": achieved, "peak": peak,
                     "peak_kind": peak_kind, "unit": "GB/s", "frac": achieved / peak,
                     "traffic": FILL_DRAM_BYTES_PER_NNZ * numh, "traffic_note": "ncu DRAM bytes per stored element "
                     "of the fill kernel on the mid system, scaled by NumH",
                     "algorithmic_bytes": int(fill_bytes)},
        "gpu_launches": launches,
        "clocks": clk,
        "e2e": e2e,
    }
    if not args.no_lsj:
        line["lsj"] = lsj_section(args, eng, sysm)
        for key, fn in (("density", density_section), ("pt2", pt2_section)):
            try:
                line[key] = fn(args, eng, sysm)
            except Exception as exc:   # an optional section must not cost the bench line
                line[key] = {"error": str(exc)[:300]}
        if "pt_block" in line.get("pt2", {}):
            line["pt2"]["pt_block"]["numh_whole"] = int(numh)

    if args.davidson_iters > 0:
        eng.form_j()
        nlv = int(sysm.params["Nlv"])
        res = eng.davidson(sysm.nd, Nlv=nlv, N_it=args.davidson_iters, Crt4=1e-8,
                           MaxNd0=int(sysm.params["MaxNd0"]), admix_crit=0.0, want_vectors=False)
        st = eng.stats()
        calls = max(1.0, st["spmm_calls"])
        spmm_ms = st["spmm_ms"] / calls
        spmm_bytes = numh * 12 + (sysm.nd + 1) * 8 + 2 * sysm.nd * nlv * 8
        sp_ach = spmm_bytes / (spmm_ms * 1e-3) / 1e9
        line["davidson"] = {
            "form": "plain FP64 (reference algorithm)", "levels": nlv, "iterations": res["iterations"],
            "ms_total": st["davidson_ms"], "ms_init": st["init_ms"],
            "ms_per_iteration": (st["davidson_ms"] - st["init_ms"]) / max(1, res["iterations"]),
            "spmm_ms_per_call": spmm_ms, "spmm_calls": int(calls),
            "max_residual": float(np.max(res["resid"])),
            "spmm_roofline": {"bound": "hbm", "achieved": sp_ach, "peak": peak, "unit": "GB/s",
                              "frac": sp_ach / peak, "algorithmic_bytes": int(spmm_bytes),
                              "storage": "lower triangle, transpose by global reductions"
                              if os.environ.get("PCI_SPMM") == "lower" or numh * 24 > 100e9
                              else "full symmetric copy"},
        }
        if not args.no_fp32_form:
            # precision form: H re-formed in FP32, FP32 SpMM, the same iterations;
            # eigenvalue difference from the FP64 form after them, per level
            eng.form_h(32)
            r32 = eng.davidson(sysm.nd, Nlv=nlv, N_it=args.davidson_iters, Crt4=1e-8, mode=1,
                               MaxNd0=int(sysm.params["MaxNd0"]), admix_crit=0.0, want_vectors=False)
            s32 = eng.stats()
            c32 = max(1.0, s32["spmm_calls"])
            sp32 = s32["spmm_ms"] / c32
            b32 = numh * 8 + (sysm.nd + 1) * 8 + 2 * sysm.nd * nlv * 4
            a32 = b32 / (sp32 * 1e-3) / 1e9
            line["davidson_fp32"] = {
                "form": "FP32 H and SpMM (FP32 accumulate); FP64 projections, eigensolve, residuals",
                "iterations": r32["iterations"],
                "ms_per_iteration": (s32["davidson_ms"] - s32["init_ms"]) / max(1, r32["iterations"]),
                "spmm_ms_per_call": sp32,
                "abs_dE_vs_fp64_per_level": [float(x) for x in np.abs(r32["Tk"] - res["Tk"])],
                "spmm_roofline": {"bound": "hbm", "achieved": a32, "peak": peak, "unit": "GB/s",
                                  "frac": a32 / peak, "algorithmic_bytes": int(b32)},
            }
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        t, n, r = cpu_sample(sysm, args.cpu_rows, 7, os.cpu_count() or 1)
        line["cpu_baseline"] = {"value": n / t, "unit": "nnz/s", "cores": os.cpu_count() or 1, "kind": "port",
                                "sample": f"{r} random rows of FormH ({n} non-zeros, {t:.1f} s), oracle "
                                          f"restatement of src/pconf.F90:1227-1290 with OpenMP"}
    if not args.no_csf:
        try:
            line["csf"] = csf_section(args, local, eng, sysm)
        except Exception as exc:   # an optional section must not cost the bench line
            line["csf"] = {"error": str(exc)[:300]}
    eng.close()
    if args.roots:
        flush = None
        torch.cuda.empty_cache()
        line["time_to_roots"] = time_to_roots(args, local, dist, peak, peak_kind)
    if args.batched:
        flush = None
        torch.cuda.empty_cache()
        line["batched"] = run_batched(args, local, rank, world, dist, peak, peak_kind)
    if rank == 0:
        print(json.dumps(line), flush=True)
    if dist is not None:
        dist.destroy_process_group()
    return 0


def lsj_section(args, eng, sysm):
    """LSJ (the kLSJ = 1 step, src/pconf.F90:2672-2962) of 10 normalised
    vectors of the configuration through pci_gpu_lsj (host call, vectors from
    host memory), against the oracle's restatement of calcLSJ on one core over
    the first configurations, scaled to all of them by calcLSJ's work per
    configuration (its determinants times the configurations after it)."""
    rng = np.random.default_rng(21)
    X = rng.standard_normal((sysm.nd, 10))
    X /= np.linalg.norm(X, axis=0)
    ts = []
    for _ in range(2):
        t0 = time.perf_counter()
        xj, xl, xs = eng.lsj(X)
        ts.append(time.perf_counter() - t0)
    out = {"workload": f"{args.config}: J, L, S of 10 normalised random vectors (Nd={sysm.nd})",
           "gpu_ms": 1e3 * ts[-1], "J_range": [float(xj.min()), float(xj.max())]}
    if not args.no_cpu_baseline:
        sys.path.insert(0, os.path.join(ROOT, "oracle"))
        import oracle as O
        o = O.Oracle(sysm)
        ndc = np.asarray(sysm.ndc, np.float64)
        w = ndc * (sysm.nc - np.arange(sysm.nc))           # calcLSJ's CompNRC checks per configuration
        k = int(np.searchsorted(np.cumsum(w), 4e8)) + 1     # about 10 s of oracle work
        k = max(1, min(k, sysm.nc))
        t0 = time.perf_counter()
        o.lsj_sums(X, 1, k)
        tc = time.perf_counter() - t0
        out["cpu_baseline"] = {"value_ms": 1e3 * tc * w.sum() / w[:k].sum(), "unit": "ms (estimate from a sample)",
                               "cores": 1, "kind": "port",
                               "sample": f"oracle calcLSJ over configurations 1..{k} of {sysm.nc} "
                                         f"({tc:.1f} s), scaled by determinants x later configurations"}
    return out


def density_section(args, eng, sysm):
    """pdtm's FormDM density pass (pci_gpu_density) for 10 normalised random
    vectors of the configuration, through the host call."""
    rng = np.random.default_rng(23)
    X = rng.standard_normal((sysm.nd, 10))
    X /= np.linalg.norm(X, axis=0)
    t0 = time.perf_counter()
    ro = eng.density(X)
    t = time.perf_counter() - t0
    tr = np.trace(ro, axis1=1, axis2=2)
    return {"workload": f"{args.config}: one-particle density matrices of 10 vectors (Nd={sysm.nd}, "
                        f"Nst={sysm.nst})", "gpu_ms": 1e3 * t,
            "trace_range": [float(tr.min()), float(tr.max())], "ne": int(sysm.ne)}


def pt2_section(args, eng, sysm):
    """conf_pt's second-order step (pci_gpu_pt2) with the first tenth of the
    determinants (whole configurations) as the CI space and 10 normalised
    random CI vectors; the rest of the list is the PT space.  First on the
    resident whole H, then on the PT block alone (pci_gpu_form_h_pt: PT rows
    against the CI columns, conf_pt's own FormH), after which the whole FP64
    H is formed again for the sections that follow."""
    cs = np.concatenate([[0], np.cumsum(sysm.ndc)])
    nd1 = int(cs[np.searchsorted(cs, sysm.nd // 10)])
    rng = np.random.default_rng(29)
    X0 = rng.standard_normal((nd1, 10))
    X0 /= np.linalg.norm(X0, axis=0)
    E = np.full(10, -50.0)                               # below every diagonal element
    t0 = time.perf_counter()
    de = eng.pt2(nd1, X0, E)
    t = time.perf_counter() - t0
    out = {"workload": f"{args.config}: CI space {nd1} determinants, PT space {sysm.nd - nd1}, 10 vectors",
           "gpu_ms": 1e3 * t, "dE_range": [float(de.min()), float(de.max())]}
    try:
        numh_pt = eng.form_h_pt(nd1, nd1)
        st = eng.stats()
        t0 = time.perf_counter()
        de_pt = eng.pt2(nd1, X0, E)
        t_pt = time.perf_counter() - t0
        out["pt_block"] = {"numh": int(numh_pt),
                           "formh_pt_ms": st["formh_ms"], "pt2_ms": 1e3 * t_pt,
                           "max_rel_dE_vs_whole": float(np.max(np.abs(de_pt - de) / np.abs(de)))}
    finally:
        eng.form_h(64)
    return out


def csf_section(args, local, e, sysm):
    """kCSF = 1 on the configuration, on the bench's engine (its matrix is
    replaced): FormH (FP64) + FormJ + jbasis/formh_sym (pci_gpu_form_csf),
    then the CSF matrix's lowest roots (the levels with 2J = Mj) to residual
    1e-8 through the batched solver; device times, form_csf host-timed."""
    from pci_b200.capi import Batch
    nlv = int(sysm.params["Nlv"])
    numh = e.form_h(64)[0]
    e.form_j()
    st = e.stats()
    t0 = time.perf_counter()
    ncsf, nnz = e.form_csf()
    t_csf = time.perf_counter() - t0
    b = Batch(local)
    b.set_value_prec(64)
    b.add_engine(e)
    r = b.davidson(nlv=nlv, max_sub=112, keep=48, max_it=400, tol=1e-8, it_per_graph=4)
    stb = b.stats()
    b.close()
    return {"workload": f"{args.config}: CSF basis (2J = Mj = {sysm.mj}), {nlv} roots to residual 1e-8",
            "ncsf": int(ncsf), "nd": int(sysm.nd), "numh_det": int(numh), "numh_csf": int(nnz),
            "formh_ms": st["formh_ms"], "formj_ms": st["formj_ms"], "form_csf_ms": 1e3 * t_csf,
            "solve_ms": stb["total_ms"], "iterations": int(r["iters"][0]), "converged": bool(r["status"][0] == 1),
            "max_residual": float(np.max(r["rnorm"])),
            "value_ms": st["formh_ms"] + st["formj_ms"] + 1e3 * t_csf + stb["total_ms"],
            "roots": [float(x) for x in r["E"][0]]}


def spmm_bytes(numh, nd, nlv, value_bytes, vec_bytes):
    """Algorithmic bytes of one lower-triangle SpMM over nlv vectors: every stored
    element (column index + value) read once, X read once, Y written once."""
    return numh * (4 + value_bytes) + (nd + 1) * 8 + 2 * nd * nlv * vec_bytes


def cpu_solve_estimate(sysm, nlv, iterations, numh, seed, threads):
    """CPU time to the roots on the host cores, from a bounded sample: the
    oracle's FormH over sampled rows (its nnz/s) and its Mxmpy over the sampled
    rows' CSR for nlv vectors (stored elements per second), scaled to the full
    matrix with the GPU run's iteration count (same algorithm and basis)."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import ctypes as C
    import oracle as O
    o = O.Oracle(sysm)
    rng = np.random.default_rng(seed)
    wins = sorted(rng.choice(np.arange(1, sysm.nd - 40), 40, replace=False))
    t0 = time.perf_counter()
    parts = [o.form_h(int(a), int(a) + 39, threads=threads) for a in wins]
    t_build = time.perf_counter() - t0
    n_build = sum(int(p[0][-1]) for p in parts)
    # Mxmpy over the sampled rows, full-length vectors, all host cores
    rows = np.concatenate([np.arange(int(a), int(a) + 40, dtype=np.int64) for a in wins])
    rp = np.concatenate([[0], np.cumsum(np.concatenate([np.diff(p[0]) for p in parts]))]).astype(np.int64)
    col = np.ascontiguousarray(np.concatenate([p[1] for p in parts]).astype(np.int32))
    val = np.ascontiguousarray(np.concatenate([p[2] for p in parts]))
    X = np.ascontiguousarray(rng.standard_normal((nlv, sysm.nd)))
    Y = np.zeros((nlv, sysm.nd))
    L = O.lib()
    f = L.orc_mxmpy_rows
    f.argtypes = [C.c_int64, C.c_int64, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_int, C.c_void_p,
                  C.c_void_p, C.c_int]
    t0 = time.perf_counter()
    reps = 0
    while time.perf_counter() - t0 < 3.0:
        f(sysm.nd, rows.size, rows.ctypes.data, rp.ctypes.data, col.ctypes.data, val.ctypes.data, nlv,
          X.ctypes.data, Y.ctypes.data, threads)
        reps += 1
    t_mx = (time.perf_counter() - t0) / reps
    build_rate = n_build / t_build
    mx_rate = col.size / t_mx
    est_s = numh / build_rate + iterations * numh / mx_rate
    return {"value_ms": 1e3 * est_s, "unit": "ms (estimate from a sample)", "cores": threads, "kind": "port",
            "formh_nnz_per_s": build_rate, "mxmpy_elements_per_s": mx_rate, "iterations": iterations,
            "sample": f"FormH of 40 windows of 40 rows ({n_build} non-zeros, {t_build:.1f} s) and Mxmpy of those "
                      f"rows for {nlv} vectors ({reps} passes), oracle restatements of src/pconf.F90:1227-1290 and "
                      f"src/davidson.f90:572-647 with OpenMP; scaled to NumH = {numh} and the GPU run's "
                      f"{iterations} iterations"}


def train_correction(args, sysm_kw, nlv, local):
    """The learned correction's network for a configuration: samples harvested
    from the solver's own converged FP64 runs of smaller systems on the same
    orbital basis at other seeds (100-103), trained on the GPU."""
    from pci_b200 import learned as LR
    from pci_b200 import system as S
    t0 = time.perf_counter()
    systems = []
    for sd in range(100, 104):
        kw = dict(sysm_kw)
        kw.update(seed=sd, max_nd=args.learn_nd)
        systems.append(S.make_system(**kw))
    F, T, info = LR.harvest(systems, nlv=nlv, rows_per_block=4000, device=local, max_sub=112, keep=48)
    model, loss = LR.train(F, T, device=local, epochs=4)
    return model, {"train_systems": f"{len(systems)} systems, seeds 100-103, {args.learn_nd} determinants each "
                                    f"(same orbital basis)", "samples": int(F.shape[0]), "loss": loss,
                   "seconds": time.perf_counter() - t0}


def time_to_roots(args, local, dist, peak, peak_kind):
    """The configuration's Nlv roots to a residual 2-norm of 1e-8 against the
    FP64 Hamiltonian through the batched solver with one block, in three
    forms, each timed as FormH + solve (device time):
      fp64           FP64 H, FP64 SpMM, diagonal correction (plain);
      mixed          FP64 H; SpMM on FP32 vectors with FP32 sums and the values rounded to
                     FP32 while every residual is above switch_tol (or until the FP32 sums
                     stop it dropping), then FP64 SpMM to the criterion;
      learned_mixed  the mixed form with the learned correction.
    Each SpMM is also set against the measured throughput of its transpose
    part's global FP64 reductions (pci_batch_probe_reduction), the limit it
    actually meets: nnz x vectors reduced words per call."""
    from pci_b200 import system as S
    from pci_b200.capi import PCI_BATCH_CORR_LEARNED, PCI_BATCH_FP64, PCI_BATCH_MIXED, Batch, Engine
    kw = S.CONFIGS[args.roots_config]()
    sysm = S.make_system(**kw)
    nlv = int(sysm.params["Nlv"])
    out = {"workload": f"{args.roots_config}: Nd={sysm.nd}, Ne={sysm.ne}, Nsu={sysm.nsu}, {nlv} roots, residual "
                       f"2-norm <= 1e-8 per root against the FP64 H",
           "metric": "time to all roots (FormH + solve), ms", "solver": "batched block Davidson, one block, "
           "subspace 112, 48 kept at a restart"}
    model = None
    if args.learned:
        model, out["learned_training"] = train_correction(args, kw, nlv, local)
    forms = [("fp64", 64, PCI_BATCH_FP64, None), ("mixed", 64, PCI_BATCH_MIXED, None)]
    if model is not None:
        forms.append(("learned_mixed", 64, PCI_BATCH_MIXED, model))
    from pci_b200.capi import probe_reduction
    red_peak = probe_reduction(local, sysm.nd, nlv)
    out["l2_reduction_peak_gbs"] = red_peak
    E = {}
    launches = 0
    for key, vp, prec, mdl in forms:
        with Engine(local) as e:
            e.load_system(sysm)
            numh, _, _ = e.form_h(64)
            st_h = e.stats()
            fh = st_h["formh_ms"]
            launches += int(st_h["formh_launches"]) + 1
            b = Batch(local)
            b.set_value_prec(vp)
            b.add_engine(e)
        kwd = dict(nlv=nlv, max_sub=112, keep=48, max_it=400, tol=1e-8, it_per_graph=4, precision=prec,
                   switch_tol=args.switch_tol)
        if mdl is not None:
            b.set_correction_model(mdl)
            kwd["correction"] = PCI_BATCH_CORR_LEARNED
        r = b.davidson(**kwd)
        st = b.stats()
        b.close()
        solve = max_over_ranks(st["total_ms"], dist, device=f"cuda:{local}")
        fh = max_over_ranks(fh, dist, device=f"cuda:{local}")
        launches += int(r["graph_launches"]) * kwd["it_per_graph"] * int(st["launches_per_iteration"])
        sp = spmm_bytes(numh, sysm.nd, nlv, 8, 8)
        ach = sp / (st["spmm_ms"] * 1e-3) / 1e9
        E[key] = r["E"][0]
        red = numh * nlv * 8 / (st["spmm_ms"] * 1e-3) / 1e9
        rec = {"value_ms": fh + solve, "formh_ms": fh, "solve_ms": solve, "iterations": int(r["iters"][0]),
               "converged": bool(r["status"][0] == 1), "max_residual": float(np.max(r["rnorm"])),
               "spmm_ms_per_call": st["spmm_ms"], "numh": int(numh),
               "spmm_roofline": {"bound": "hbm", "kernel": "SpMM, FP64 vectors", "achieved": ach, "peak": peak,
                                 "peak_kind": peak_kind, "unit": "GB/s", "frac": ach / peak,
                                 "algorithmic_bytes": int(sp)},
               "spmm_l2_reduction": {"bound": "L2 reductions", "achieved": red, "peak": red_peak,
                                     "peak_kind": "measured (pci_batch_probe_reduction)", "unit": "GB/s",
                                     "frac": red / red_peak, "reduced_bytes": int(numh * nlv * 8)}}
        if prec == PCI_BATCH_MIXED:
            sp32 = spmm_bytes(numh, sysm.nd, nlv, 4, 4)
            a32 = sp32 / (st["spmm32_ms"] * 1e-3) / 1e9
            rec.update(fp32_iterations=int(st["fp32_iterations"]), spmm32_ms_per_call=st["spmm32_ms"],
                       spmm32_roofline={"bound": "hbm", "kernel": "SpMM, FP32 vectors and hi values", "achieved": a32,
                                        "peak": peak, "peak_kind": peak_kind, "unit": "GB/s", "frac": a32 / peak,
                                        "algorithmic_bytes": int(sp32)})
        out[key] = rec
    for key in E:
        if key != "fp64":
            out[f"abs_dE_{key}_vs_fp64_per_root"] = [float(x) for x in np.abs(E[key] - E["fp64"])]
            out[f"speedup_{key}_vs_fp64"] = out["fp64"]["value_ms"] / out[key]["value_ms"]
    if model is not None:
        model.close()
    out["gpu_launches"] = launches
    if not args.no_cpu_baseline:
        out["cpu_baseline"] = cpu_solve_estimate(sysm, nlv, out["fp64"]["iterations"], out["fp64"]["numh"], 11,
                                                 os.cpu_count() or 1)
    return out


TUNE_CACHE = os.path.join(os.environ.get("XDG_CACHE_HOME") or os.path.join(os.path.expanduser("~"), ".cache"),
                          "pci_b200", "spmm_tune_cache.txt")


def tune_cache_path(path):
    """The SpMM tuning cache file (its folder created); '' disables the cache."""
    if not path:
        return None
    os.makedirs(os.path.dirname(os.path.abspath(path)), exist_ok=True)
    return path


def run_batched(args, local, rank, world, dist, peak, peak_kind):
    """The batched form: 64 synthetic ions (seeds 1000-1063; 2-4 valence
    electrons, 30-120 orbitals, mixed M and parity, 2k-400k determinants
    log-uniform), each H built on the device in FP32 and handed to one batch,
    6 roots per block to a residual of 1e-8, every block in the same
    graph-replayed launches."""
    from pci_b200 import system as S
    from pci_b200.capi import Batch, Engine
    blocks = S.make_batch(args.batch_blocks)
    # with several GPUs the blocks are split over the ranks (largest first to
    # the least loaded rank by determinants), no communication
    order = S.split_blocks([blk.nd for blk in blocks], world, rank)
    b = Batch(local)
    formh_ms = 0.0
    launches = 0
    numh_blk = []
    for i in order:
        with Engine(local) as e:
            e.load_system(blocks[i])
            numh_blk.append(e.form_h(32)[0])
            st = e.stats()
            formh_ms += st["formh_ms"]
            launches += int(st["formh_launches"]) + 1
            b.add_engine(e)
    nblk, rows, nnz = b.info()
    nlv = 6
    if args.batch_variant >= 0:
        variant, tune_ms, cached = args.batch_variant, None, False
    else:
        variant, tune_ms, cached = b.tune(nlv, tune_cache_path(args.tune_cache))
    # subspace 64 with 24 kept at a restart: measured 6.5 s against 7.1 s for
    # 48/12 and 7.7 s for 36/12 on this workload (fewer iterations)
    r = b.davidson(nlv=nlv, max_sub=64, keep=24, max_it=300, tol=1e-8, it_per_graph=4, spmm_variant=variant)
    st = b.stats()
    b.close()
    solve_ms = max_over_ranks(st["total_ms"], dist, device=f"cuda:{local}")
    formh_ms = max_over_ranks(formh_ms, dist, device=f"cuda:{local}")
    sp_bytes = nnz * 8 + rows * 12 + 2 * rows * nlv * 8
    sp_ach = sp_bytes / (st["spmm_ms"] * 1e-3) / 1e9
    lanes, per_sm = [(s_, c_) for s_ in (32, 16, 8) for c_ in (4, 8, 16, 32)][variant]
    launches += r["graph_launches"] * 4 * int(st["launches_per_iteration"])
    out = {
        "workload": f"{len(blocks)} blocks (seeds 1000-{1000 + len(blocks) - 1}); on rank 0: {nblk} blocks, "
                    f"{rows} determinants, {nnz} stored elements (FP32 values, int32 columns), {nlv} roots "
                    f"per block",
        "parallelism": f"blocks split over {world} GPU(s), no communication" if world > 1 else "one GPU",
        "metric": "time to all roots at residual <= 1e-8 (H-build + solve)",
        "value_ms": formh_ms + solve_ms, "formh_ms": formh_ms, "solve_ms": solve_ms,
        "solve_setup_ms": st["setup_ms"], "n_gpus": world,
        "converged_blocks": int(np.sum(r["status"] == 1)),
        "max_residual": float(np.max(r["rnorm"])),
        "iterations_max": int(np.max(r["iters"])), "iterations_median": float(np.median(r["iters"])),
        "graph_launches": int(r["graph_launches"]), "kernels_per_iteration": int(st["launches_per_iteration"]),
        "spmm_ms_per_call": st["spmm_ms"], "subspace": {"max": 64, "kept_at_restart": 24},
        "storage": "lower triangles, transpose part by global reductions",
        "spmm_variant": {"index": variant, "lanes_per_row": lanes, "blocks_per_sm": per_sm,
                         "from_cache": cached, "tuned_ms": tune_ms},
        "spmm_roofline": {"bound": "hbm", "kernel": "kb_spmm", "achieved": sp_ach, "peak": peak,
                          "peak_kind": peak_kind, "unit": "GB/s", "frac": sp_ach / peak,
                          "algorithmic_bytes": int(sp_bytes)},
        "gpu_launches": launches,
    }
    if not args.no_cpu_baseline and rank == 0 and world == 1:
        # the oracle's FormH and Mxmpy rates on the largest block, applied to
        # every block's stored elements and iteration count (blocks in sequence)
        try:
            big = int(np.argmax(numh_blk))
            rates = cpu_solve_estimate(blocks[order[big]], nlv, 1, numh_blk[big], 17, os.cpu_count() or 1)
            est_s = sum(nh / rates["formh_nnz_per_s"] + int(r["iters"][j]) * nh / rates["mxmpy_elements_per_s"]
                        for j, nh in enumerate(numh_blk))
            out["cpu_baseline"] = {"value_ms": 1e3 * est_s, "unit": "ms (estimate from a sample)",
                                   "cores": rates["cores"], "kind": "port",
                                   "sample": "the largest block's " + rates["sample"].split(";")[0] + "; its "
                                             "rates applied to every block's stored elements and iteration count, "
                                             "the blocks solved one after another"}
        except Exception as exc:   # the estimate must not cost the bench line
            out["cpu_baseline"] = {"error": str(exc)[:300]}
    return out


def run_profile_case(args):
    """A short batched solve for profiler captures: the configuration's FP64 H
    built on the device, then args.case_iters iterations of the batched solver
    with the learned correction (a freshly initialised network), so every
    kernel of an iteration (SpMM, tensor-core Gram products, tensor-core
    network) runs."""
    from pci_b200 import learned as LR
    from pci_b200 import system as S
    from pci_b200.capi import PCI_BATCH_CORR_LEARNED, Batch, Engine, Mlp
    sysm = S.make_system(**S.CONFIGS[args.profile_case]())
    m = Mlp(LR.NIN_DEFAULT, 0, seed=1)
    if args.case_train > 0:   # training steps on random samples (the network's tensor-core GEMMs)
        rng = np.random.default_rng(5)
        F = rng.standard_normal((16384, LR.NIN_DEFAULT)).astype(np.float32)
        T = rng.standard_normal(16384).astype(np.float32)
        m.train(F, T, epochs=args.case_train, batch=4096, lr=1e-3, seed=1)
    with Engine(0) as e:
        e.load_system(sysm)
        e.form_h(64)
        b = Batch(0)
        b.set_value_prec(64)
        b.add_engine(e)
    b.set_correction_model(m)
    r = b.davidson(nlv=int(sysm.params["Nlv"]), max_sub=96, keep=48, max_it=args.case_iters, tol=1e-8,
                   correction=PCI_BATCH_CORR_LEARNED, spmm_variant=0)
    print(json.dumps({"profile_case": args.profile_case, "Nd": sysm.nd, "iterations": int(r["iters"][0]),
                      "stats": b.stats()}), flush=True)
    b.close()
    m.close()
    return 0


def main():
    args = parse()
    if args.profile_case:
        return run_profile_case(args)
    if args.tune_cache is None:
        args.tune_cache = TUNE_CACHE
    if args.impl == "reference":
        return run_reference(args)
    return run_ours(args)


if __name__ == "__main__":
    sys.exit(main())
