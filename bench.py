"""Benchmark of the droplet update path (particle-updates/s) on B200.

Headline workload (N = 1): a 256^3 periodic field and 1,000,000 droplets with radii
uniform in [10, 40] um, the mixed-precision path as the measured value and the FP64 path
beside it.  One "step" is one droplet substep of the update path: interpolation of the
three velocity components, history, drag advance, position update, periodic wrap and the
PERIODIC reorder (plus the amortised spatial re-sort of the device order).  Inputs (field,
droplet state) are resident in HBM when the timed region starts and are larger than L2
(field 218 MB FP32 / 441 MB FP64, droplet state ~0.2 GB), so no L2 flush is needed.
N > 1 runs independent replicas, one per GPU (the path does not shard on one node; weak
scaling).

After the timed region the line gathers the other workloads of the benchmark set, each a
seeded synthetic stand-in with the stated shapes:

* ``full_step``: the coupled 256^3 flow + 1M-droplet step with HDI (device and end-to-end);
* ``config0``: 64^3 deterministic forcing, 500 steps, 20,000 droplets of 20 um at
  St_eta = 0.5, Sv = 1: RDF and w_r at contact and the collision count, FP64 and mixed;
* ``config1``: 128^3 OU forcing, 2000 steps, 100,000 droplets of 20/30 um: pair lists of
  both paths checked against the oracle's detection on identical inputs at sampled steps
  (the reference's 128^3 stochastic parameter set: nu 0.0945, dt 1e-4);
* ``adjoint``: 128^3 field after 300 forced FP64 steps, 200,000 droplets of 25 um, 400
  substeps checkpointed every 20: forward/backward cost, central differences (h = 1e-6) on
  sampled entries of tau_p, x_0 and u, mixed-vs-FP64 gradient error;
* ``config4``: 512^3 / 5M lognormal droplets with HDI and coalescence: step breakdown
  (FFT, flow kernels, interpolation, advance, cell list, collision, HDI) and GB/s;
* ``cpu_baseline``: the FP64 CPU oracle timed on this host's cores, which is also the
  checker of the GPU outputs above (``errors_vs_fp64_oracle``, config-0 and config-1
  oracle values).  Nothing is timed while the oracle runs on the GPU's behalf.

``--impl reference`` times the CPU restatement of the reference's path (the Fortran/MPI
reference itself cannot be built here) on this host's cores on a bounded sample.
"""
from __future__ import annotations

import argparse
import json
import math
import os
import re
import statistics
import subprocess
import sys
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

N_GRID = 256
N_PART = 1_000_000
SETS_UM = [10.0, 20.0, 30.0, 40.0]
PHYS = dict(dt=5e-4, rnu=8e-4, etk_dns=0.0079, tauk_dns=0.078)
CONFIG = {"workload": "256^3 field, 1,000,000 droplets, radii U[10,40] um, update substep",
          "grid": N_GRID, "droplets": N_PART, "precision": "mixed (FP32 arithmetic, FP64 positions)",
          "l2": "no flush: inputs larger than L2 (FP32 field 218 MB + droplet state ~0.2 GB)",
          "parallelism": "replicas"}
ERR_STEPS = 10
C0 = dict(n=64, npart=20_000, radius_um=20.0, nu=0.0025, dt=1e-3, steps=500, ediss_cloud=1554.0,
          gravity=771.0, seed=1234)
# the reference's own 128^3 stochastic-forcing set (parameter.d_128_stoch): with its OU forcing
# amplitude (flowlib.f90:401-402) the flow leaves AB2's stable range at dt = 8e-4 and 4e-4
C1 = dict(n=128, npart=100_000, radius_um=[20.0, 30.0], nu=0.09449408, dt=1e-4, etk_dns=0.02189,
          tauk_dns=0.005072, steps=2000, samples=40, iseedf=232300, seed=1234)
ADJ = dict(n=128, np=200_000, radius_um=25.0, nsteps=400, checkpoint_every=20, dt=5e-4, spinup=300,
           spin_nu=0.0025, spin_dt=1e-3, pair_factor=2.0, fd_h=1e-6, fd_entries=10, seed=1234)
C4 = dict(n=512, npart=5_000_000, nu=3e-4, dt=5e-4, etk_dns=0.00484, tauk_dns=0.078, lognormal=(25.0, 0.3),
          clip_um=(10.0, 60.0))


def _dist():
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return ws, rank, local


def max_over_ranks(values, ws, device="cpu"):
    """Element-wise max of per-rank timings (the replica run's device times; every rank
    takes this collective at the same point)."""
    import torch
    t = torch.tensor([float(v) for v in values], dtype=torch.float64, device=device)
    if ws > 1:
        import torch.distributed as dist
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return [float(x) for x in t.tolist()]


def replica_value(ws, npart, ms_per_step):
    """Whole-job particle-updates/s of ws replicas, each updating npart droplets per step."""
    return ws * npart / (ms_per_step * 1e-3)


def _clock_sampler(dev: int):
    cmd = ["nvidia-smi", f"--id={dev}",
           "--query-gpu=clocks.sm,clocks.max.sm,clocks_event_reasons.hw_slowdown,"
           "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
           "clocks_event_reasons.sw_power_cap", "--format=csv,noheader,nounits", "-lms", "200"]
    try:
        return subprocess.Popen(cmd, stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
    except OSError:
        return None


def _clock_summary(proc):
    if proc is None:
        return None
    proc.terminate()
    try:
        out, _ = proc.communicate(timeout=5)
    except subprocess.TimeoutExpired:
        proc.kill()
        out, _ = proc.communicate()
    sm, mx, reasons = [], [], set()
    names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
    for line in out.strip().splitlines():
        f = [x.strip() for x in line.split(",")]
        if len(f) < 6:
            continue
        try:
            sm.append(float(f[0])); mx.append(float(f[1]))
        except ValueError:
            continue
        for nm, v in zip(names, f[2:6]):
            if v.lower().startswith("active"):
                reasons.add(nm)
    if not sm:
        return None
    return {"sm_mhz": statistics.median(sm), "sm_max_mhz": max(mx), "reasons": sorted(reasons),
            "samples": len(sm)}


def _peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        d = json.load(open(p))
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def _profile_traffic():
    """DRAM bytes per update step of the two update kernels from the committed ncu summary."""
    p = os.path.join(ROOT, "profiles", "update_kernels_mixed_256_1M.md")
    if not os.path.exists(p):
        return None
    m = re.search(r"traffic_bytes_per_step:\s*([0-9.eE+]+)", open(p).read())
    return float(m.group(1)) if m else None


def _gbs(nbytes, ms):
    return nbytes / (ms * 1e-3) / 1e9 if ms and ms > 0 else None


def _make(precision, dev, npart=N_PART, n=N_GRID, hdi=False):
    from mpi_2d_domain_decomp_turb_particles_b200 import Partlib, ParticleParams
    from mpi_2d_domain_decomp_turb_particles_b200.synthetic import droplets
    p = ParticleParams(nx=n, npart=npart, radius_um=SETS_UM, precision=precision, device=dev,
                       new_particle=True, hdi_included=hdi, nonoverlap=hdi, hdi_trunc=50.0, **PHYS)
    g = Partlib(p)
    g.part_init()
    s = g.scalars()
    scale = s.radius[0] / SETS_UM[0]
    yp = droplets(npart, scale, radius_um=(10.0, 40.0), seed=290710 + 17 * dev)
    g.set_particles(yp)
    return g


def _time_update(g, stream, steps, warmup, torch):
    """(ms per step by events around the loop, update-kernel ms per step, launches,
    interpolation-kernel ms, advance-kernel ms)."""
    for _ in range(warmup):
        g.update_step()
    g.sync()
    g.timing(reset=True)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    e0.record(stream)
    for _ in range(steps):
        g.update_step()
    e1.record(stream)
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1)
    ims, ams = g.timing_split()
    kms, nk, launches = g.timing(reset=True)
    return ms / steps, kms, launches, ims, ams


def _dissipation_scales(u, nu):
    """(epsilon, eta, tau_eta) of a periodic 2 pi velocity field u (3, n, n, >=n) from its
    spectrum: epsilon = nu <du_i/dx_j du_i/dx_j> (homogeneous flow)."""
    import numpy as np
    n = u.shape[1]
    k = np.fft.fftfreq(n, 1.0 / n)
    kr = np.fft.rfftfreq(n, 1.0 / n)
    KZ, KY, KX = np.meshgrid(k, k, kr, indexing="ij")
    k2 = KX * KX + KY * KY + KZ * KZ
    w = np.where((KX == 0) | (KX == n // 2), 1.0, 2.0)
    eps = 0.0
    for c in range(3):
        uh = np.fft.rfftn(np.asarray(u[c][:, :, :n])) / n ** 3
        eps += float((w * k2 * np.abs(uh) ** 2).sum())
    eps *= nu
    return eps, (nu ** 3 / eps) ** 0.25, (nu / eps) ** 0.5


def _shell_energies(uh):
    """Energies of shells 1 and 2 of the flow's spectral velocity (kx = 0 modes count half;
    the convention of the deterministic forcing, flowlib.f90:195-229)."""
    import numpy as np
    n = uh.shape[1]
    e = [0.0, 0.0]
    for kz in range(-2, 3):
        for ky in range(-2, 3):
            for kx in range(0, 3):
                sh = int(math.sqrt(kx * kx + ky * ky + kz * kz) + 0.5)
                if sh not in (1, 2):
                    continue
                t = float(np.sum(np.abs(uh[:, kz % n, ky % n, kx]) ** 2))
                e[sh - 1] += 0.5 * t if kx == 0 else t
    return e


def _det_flow(n, nu, dt, seed, dev, torch):
    """Flow started from the seeded spectrum with the deterministic forcing holding the
    energies of shells 1 and 2 at their initial values; returns (flow, initial velocity)."""
    from mpi_2d_domain_decomp_turb_particles_b200.flow import Flow
    from mpi_2d_domain_decomp_turb_particles_b200.synthetic import spectral_field
    u0 = torch.stack(spectral_field(n, seed=seed, device=f"cuda:{dev}")).contiguous()
    probe = Flow(n, nu, dt, forcing=0, device=dev)
    probe.set_velocity(u0)
    e1, e2 = _shell_energies(probe.spectral()[0])
    probe.close()
    fl = Flow(n, nu, dt, forcing=1, force=(e1, e2), device=dev)
    fl.set_velocity(u0)
    return fl, u0


NEAR = 20   # RDF bins 0..19: separations in [R, 2R), R = a_i + a_j (bin width 0.05 R)


def _rdf_expected(npart, rc, steps):
    """Pairs per RDF bin expected over `steps` steps for uniform droplets (monodisperse,
    contact distance rc; bins of 0.05 rc from rc, partlib.f90:1641-1657)."""
    import numpy as np
    r = rc * (1 + 0.05 * np.arange(181))
    shell = 4.0 / 3.0 * np.pi * (r[1:] ** 3 - r[:-1] ** 3)
    return 0.5 * npart * (npart / (2 * math.pi) ** 3) * shell * steps


def _rdf_summary(nir, wr, expect):
    """RDF and mean w_r at contact (bin 0) and near contact (bins 0..NEAR-1)."""
    n0, nn = float(nir[0]), float(nir[:NEAR].sum())
    return {"rdf_contact": n0 / expect[0], "wr_contact": float(wr[0]) / n0 if n0 else None,
            "rdf_near_contact": nn / float(expect[:NEAR].sum()),
            "wr_near_contact": float(wr[:NEAR].sum()) / nn if nn else None,
            "pairs_bin0": int(n0), "pairs_near_contact": int(nn), "pairs_all_bins": int(nir.sum()),
            "nirbin": nir}


def _field_sum(ts):
    return float(sum(float(t.double().sum()) for t in ts))


class _Hist:
    """Sums of the RDF counts (nirbin) and w_r sums (wrbin) over every step: the written
    histograms at each 5-step boundary (the accumulators restart there, partlib.f90:
    1659-1718) plus what is left in the accumulators at the end."""

    def __init__(self):
        self.nir = 0
        self.wr = 0

    def gpu_step(self, x, rep):
        if rep.written:
            h = x.histograms(written=True)
            self.nir = self.nir + h["nirbin"].astype("float64")
            self.wr = self.wr + h["wrbin"]

    def gpu_end(self, x):
        h = x.histograms(written=False)
        self.nir = self.nir + h["nirbin"].astype("float64")
        self.wr = self.wr + h["wrbin"]

    def oracle_step(self, o):
        if o.geti("written"):
            self.nir = self.nir + o.hist("out_nirbin").astype("float64")
            self.wr = self.wr + o.hist("out_wrbin")

    def oracle_end(self, o):
        self.nir = self.nir + o.hist("nirbin").astype("float64")
        self.wr = self.wr + o.hist("wrbin")


# ---------------------------------------------------------------------------------------
# GPU legs
# ---------------------------------------------------------------------------------------
def run_ours(args):
    import torch
    import torch.distributed as dist
    from mpi_2d_domain_decomp_turb_particles_b200.bytes_model import (advance_bytes, collision_bytes, interp_bytes,
                                                                      interp_onchip, update_bytes)

    ws, rank, local = _dist()
    if ws > 1:
        dist.init_process_group("nccl", init_method="env://", timeout=__import__("datetime").timedelta(seconds=300))
    torch.cuda.set_device(local)
    dev = local
    from mpi_2d_domain_decomp_turb_particles_b200.synthetic import spectral_field
    field = spectral_field(N_GRID, seed=1234, device=f"cuda:{dev}")
    stream = torch.cuda.Stream(device=dev)

    # ---- mixed path (the measured value) ----
    g = _make("mixed", dev)
    g.set_stream(stream)
    g.set_fields(*field)
    g.sync()
    clk = _clock_sampler(dev) if rank == 0 else None
    time.sleep(0.4)   # the sampler's first reading lands before the timed region
    if ws > 1:
        dist.barrier()
    ms_step, kernel_ms, launches, interp_ms, adv_ms = _time_update(g, stream, args.steps, args.warmup, torch)
    clocks = _clock_summary(clk)
    nsm = torch.cuda.get_device_properties(dev).multi_processor_count
    ms_step, kernel_ms = max_over_ranks([ms_step, kernel_ms], ws, device=f"cuda:{dev}")
    value = replica_value(ws, N_PART, ms_step)

    # ---- full particle substep (cell lists, collision detection and statistics) ----
    full = []
    cand = 0
    for _ in range(3):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        c, _gm = g.particle_step()
        e1.record(stream)
        torch.cuda.synchronize()
        full.append(e0.elapsed_time(e1))
        cand = c.candidate_pairs
    full_ms = statistics.median(full)
    coll_ms = g.phase_times()[2]

    # ---- end to end through the C ABI with host buffers (pinned) ----
    host = [f.cpu().pin_memory() for f in field]
    # newly pinned pages upload slower for the first few dozen copies (46 against 55 GB/s
    # measured on a B200 host), so the warm-up runs at least five steps (15 uploads)
    e2e_steps = max(1, min(args.steps, 10))
    for _ in range(max(5, args.warmup)):
        g.set_fields(*[h.numpy() for h in host]); g.update_step(); g.mean_vel()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(e2e_steps):
        g.set_fields(*[h.numpy() for h in host])    # H2D of the step's field (INTERPOLATE(v, icpt))
        g.update_step()
        mv = g.mean_vel()                            # D2H of the step's statistic (MEAN_VEL)
    e1.record(stream)
    torch.cuda.synchronize()
    e2e_ms = e0.elapsed_time(e1) / e2e_steps
    h2d = sum(h.numel() * h.element_size() for h in host)
    d2h = mv.nbytes
    g.close()
    del g, host

    # ---- FP64 path, same workload ----
    g64 = _make("fp64", dev)
    g64.set_stream(stream)
    g64.set_fields(*field)
    g64.sync()
    ms64, kms64, _, ims64, ams64 = _time_update(g64, stream, max(3, args.steps // 2), args.warmup, torch)
    g64.close()
    (ms64,) = max_over_ranks([ms64], ws, device=f"cuda:{dev}")
    value64 = replica_value(ws, N_PART, ms64)

    rec = {}
    extra = {}
    if rank == 0:
        rec["errors"] = errors_gpu(dev, torch, field)
        extra["full_step"] = full_step_bench(dev, torch, field) if not args.no_full else None
        host_field = [f.cpu().numpy() for f in field]
        del field
        torch.cuda.empty_cache()
        if not args.no_configs:
            rec["config0"] = config0_gpu(dev, torch)
            rec["config1"] = config1_gpu(dev, torch)
        extra["adjoint"] = adjoint_bench(dev, torch) if not args.no_adjoint else None
        c4 = None
        if not args.no_config4:
            try:
                c4 = config4_bench(dev, torch)
            except Exception as ex:   # reported, not fatal: the headline numbers stand alone
                c4 = {"error": f"{type(ex).__name__}: {ex}"}
        extra["config4"] = c4
    else:
        del field

    if rank == 0:
        peak, kind = _peaks()
        alg = update_bytes("mixed", N_GRID, N_PART)
        achieved = alg / (kernel_ms * 1e-3) / 1e9
        alg64 = update_bytes("fp64", N_GRID, N_PART)
        frac64 = _gbs(alg64, kms64) / peak
        traffic = _profile_traffic()
        cpu = cpu_baseline(rec, host_field)
        line = {
            "metric": "particle-updates/s (256^3, 1M droplets, mixed precision)",
            "value": value, "unit": "particle-updates/s", "n_gpus": ws, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms_step, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32 (positions f64)", "data": "synthetic (seeded spectrum field, uniform droplets)",
            "config": CONFIG,
            "fp64_value": value64, "fp64_ms_per_step": ms64, "mixed_over_fp64": value / value64,
            "mixed_roofline_frac": achieved / peak, "fp64_roofline_frac": frac64,
            "byte_ratio_fp64_over_mixed": alg64 / alg,
            "kernels": {
                "mixed": {"interp_ms": interp_ms, "advance_ms": adv_ms,
                          "interp_gbs": _gbs(interp_bytes("mixed", N_GRID, N_PART), interp_ms),
                          "advance_gbs": _gbs(advance_bytes("mixed", N_GRID, N_PART), adv_ms),
                          "interp_onchip": interp_onchip("mixed", N_PART, interp_ms, nsm, clocks)},
                "fp64": {"update_kernels_ms": kms64, "interp_ms": ims64, "advance_ms": ams64,
                         "interp_gbs": _gbs(interp_bytes("fp64", N_GRID, N_PART), ims64),
                         "advance_gbs": _gbs(advance_bytes("fp64", N_GRID, N_PART), ams64),
                         "interp_onchip": interp_onchip("fp64", N_PART, ims64, nsm, clocks),
                         "algorithmic_bytes": alg64}},
            "full_step_ms": full_ms, "collision_ms": coll_ms,
            "collision_candidate_pairs_per_s": cand / (coll_ms * 1e-3) if coll_ms > 0 else None,
            "collision_roofline": {"algorithmic_bytes": collision_bytes("mixed", N_PART),
                                   "achieved_gbs": _gbs(collision_bytes("mixed", N_PART), coll_ms),
                                   "frac": _gbs(collision_bytes("mixed", N_PART), coll_ms) / peak,
                                   "candidate_pairs": cand,
                                   "note": "COLLISION_DET phase (search + evaluation + host bookkeeping); "
                                           "latency-bound cell search, bytes a lower bound"},
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": achieved / peak, "traffic": traffic, "peak_kind": f"{kind} (burst copy)",
                         "kernel": "k_interp_col + k_advance_fused, per update step",
                         "algorithmic_bytes": alg, "kernel_ms": kernel_ms},
            "e2e": {"value": N_PART / (e2e_ms * 1e-3), "unit": "particle-updates/s",
                    "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h,
                    "path": "dl_set_field (host FP64 field, pinned) + dl_update_step + dl_mean_vel"},
            "e2e_coupled": (extra["full_step"] or {}).get("e2e"),
            "errors_vs_fp64_oracle": cpu.pop("errors", None),
            "full_step": extra["full_step"],
            "config0": cpu.pop("config0", None),
            "config1": cpu.pop("config1", None),
            "config4": extra["config4"],
            "adjoint": extra["adjoint"],
            "gpu_launches": int(launches),
            "clocks": clocks,
            "cpu_baseline": cpu,
        }
        print(json.dumps(line), flush=True)
    if ws > 1:
        dist.barrier()
        dist.destroy_process_group()


def full_step_bench(dev, torch, field):
    """The whole time step of the headline configuration: the device flow step (256^3 FP64
    pseudo-spectral, stochastic forcing) and the droplet substep with hydrodynamic
    interaction (1M droplets, radii U[10, 40] um, mixed precision), device time per step;
    and the same step end to end through the public calls (host clock around each step,
    the step's reports read back to the host; no host inputs: the field never leaves HBM)."""
    import numpy as np
    from mpi_2d_domain_decomp_turb_particles_b200.flow import Flow
    fl = Flow(N_GRID, PHYS["rnu"], PHYS["dt"], forcing=2, iseedf=232300, device=dev)
    u = torch.stack(field).contiguous()
    fl.set_velocity(u)
    del u
    stream = torch.cuda.Stream(device=dev)
    fl.set_stream(stream)
    for _ in range(3):
        fl.step()
    fl.timing(True)
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    nf = 10
    e0.record(stream)
    for _ in range(nf):
        fl.step()
    e1.record(stream)
    torch.cuda.synchronize()
    flow_ms = e0.elapsed_time(e1) / nf
    fparts = fl.timing(False)
    # droplets with HDI, fed by the flow
    g = _make("mixed", dev, hdi=True)
    g.set_stream(stream)
    fl.step(g)
    g.periodic()
    g.overlap_det()
    g.sync()
    for _ in range(2):
        fl.step(g)
        g.particle_step()
    torch.cuda.synchronize()
    ts, iters, phases = [], [], []
    for _ in range(5):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        fl.step(g)
        _c, gm = g.particle_step()
        e1.record(stream)
        torch.cuda.synchronize()
        ts.append(e0.elapsed_time(e1))
        iters.append(gm.iterations)
        phases.append(g.phase_times())
    # end to end: host wall clock per coupled step, reports to the host each step
    wall = []
    for _ in range(5):
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        fl.step(g)
        c, gm = g.particle_step()
        mv = g.mean_vel()
        wall.append(time.perf_counter() - t0)
    ph = np.median(np.array(phases), axis=0)
    g.close()
    fl.close()
    e2e_s = statistics.median(wall)
    return {"workload": "256^3 FP64 flow step (stochastic forcing) + 1M-droplet substep with HDI (50 radii), mixed",
            "flow_step_ms": flow_ms, "step_ms": statistics.median(ts),
            "flow_parts_ms": fparts,
            "particle_phase_ms": {"interp_fvp": ph[0], "interp_kernel": ph[7], "cell_list": ph[1],
                                  "hdi": ph[3], "advance": ph[6], "collision": ph[2],
                                  "periodic_relocate": ph[4], "overlap": ph[5]},
            "gmres_iterations": iters,
            "e2e": {"value": N_PART / e2e_s, "unit": "particle-updates/s (coupled flow + HDI step)",
                    "step_ms": e2e_s * 1e3, "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": int(mv.nbytes) + 64,
                    "path": "dl_flow_step(flow, droplets) + dl_particle_step + dl_mean_vel, host clock per step"}}


def errors_gpu(dev, torch, field, steps=ERR_STEPS):
    """The mixed and FP64 paths on identical headline inputs (1M droplets in the 256^3
    field): interpolated velocity at identical positions, then `steps` full particle steps
    (collision detection and statistics on).  Returns what the oracle leg compares."""
    import numpy as np
    g = {p: _make(p, dev) for p in ("mixed", "fp64")}
    out = {"yp0": g["fp64"].get_particles()["yp"].copy(), "steps": steps,
           "radius_sets": np.array(g["fp64"].scalars().radius[:len(SETS_UM)])}
    for p, x in g.items():
        x.set_fields(*field)
        x.prepare_interp()
        for k in (1, 2, 3):
            x.interpolate(None, k)
        r = {"vp": x.get_particles()["vp"].copy(), "icc": [], "wr": [], "pairs": []}
        hist = _Hist()
        for _ in range(steps):
            rep, _gm = x.particle_step()
            r["icc"].append(list(rep.icc[:]))
            hist.gpu_step(x, rep)
            r["wr"].append(x.contacts()[1][:, 11].copy() if rep.ncontact else np.zeros(0))
            r["pairs"].append(sorted(map(tuple, x.pairs().tolist())))
        hist.gpu_end(x)
        r["nirbin"], r["wrbin"] = hist.nir, hist.wr
        r["yp"] = x.get_particles()["yp"].copy()
        out[p] = r
        x.close()
    return out


def config0_gpu(dev, torch):
    """64^3, nu = 0.0025, deterministic forcing of shells 1 and 2, dt = 1e-3, 500 steps;
    20,000 droplets of 20 um placed uniformly (PART_INIT), starting at the interpolated fluid
    velocity; St_eta = 0.5 and Sv = 1 from the field's initial dissipation.  Both precisions
    step in the same flow; per-step histograms and collision counts are kept for the
    RDF at contact, w_r at contact and the collision count."""
    import numpy as np
    from mpi_2d_domain_decomp_turb_particles_b200 import Partlib, ParticleParams
    n = C0["n"]
    fl, u0 = _det_flow(n, C0["nu"], C0["dt"], C0["seed"], dev, torch)
    eps, eta, tau = _dissipation_scales(u0.cpu().numpy(), C0["nu"])
    del u0
    stream = torch.cuda.Stream(device=dev)
    fl.set_stream(stream)
    params = dict(nx=n, npart=C0["npart"], radius_um=[C0["radius_um"]], dt=C0["dt"], rnu=C0["nu"],
                  etk_dns=eta, tauk_dns=tau, ediss_cloud=C0["ediss_cloud"], gravity=C0["gravity"],
                  init_velocity=1, device=dev)
    g = {}
    for p in ("fp64", "mixed"):
        g[p] = Partlib(ParticleParams(precision=p, **params))
        g[p].part_init()
        g[p].set_stream(stream)
    s = g["fp64"].scalars()
    a = s.radius[0]
    st = s.tau_cloud_const2 * a * a / tau
    sv = s.sv_const * a * a / (eta / tau)
    acc = {p: {"coll": 0, "hist": _Hist()} for p in g}
    sums = []
    t0 = time.perf_counter()
    for _ in range(C0["steps"]):
        fl.step()
        vt = fl.velocity_tensors()
        sums.append(_field_sum(vt))
        for p, x in g.items():
            x.set_fields(*vt)
            rep, _ = x.particle_step()
            acc[p]["hist"].gpu_step(x, rep)
            acc[p]["coll"] += int(sum(rep.icc[:]))
    wall = time.perf_counter() - t0
    for p, x in g.items():
        acc[p]["hist"].gpu_end(x)
        x.close()
    fl.close()
    npart = C0["npart"]
    expect = _rdf_expected(npart, 2 * a, C0["steps"])
    res = {"workload": "64^3 deterministic forcing (shells 1, 2), nu 0.0025, dt 1e-3, 500 steps; 20,000 droplets "
                       "of 20 um, initial velocity = fluid velocity",
           "epsilon": eps, "eta": eta, "tau_eta": tau, "st_eta": st, "sv": sv, "field_sums": sums,
           "wall_s": wall, "expected_pairs": {"bin0": expect[0], "near_contact": float(expect[:NEAR].sum())}}
    for p in g:
        res[p] = _rdf_summary(acc[p]["hist"].nir[:, 0, 0], acc[p]["hist"].wr[:, 0, 0], expect)
        res[p]["collisions"] = acc[p]["coll"]
    return res


def config1_gpu(dev, torch):
    """128^3 OU forcing (the reference's 128^3 stochastic set: nu = 0.0945, dt = 1e-4, DNS
    Kolmogorov scales 0.02189 / 0.005072), 2000 steps; 100,000 droplets of 20 and 30 um
    (50/50, PART_INIT).  Both precisions step in the same flow; at `samples` evenly
    spaced steps each path runs the step through the separate entry points and keeps its
    state right before COLLISION_DET and what its detection returned, for the oracle to
    detect again on identical inputs."""
    import numpy as np
    from mpi_2d_domain_decomp_turb_particles_b200 import Partlib, ParticleParams
    from mpi_2d_domain_decomp_turb_particles_b200.flow import Flow
    from mpi_2d_domain_decomp_turb_particles_b200.synthetic import spectral_field
    n, steps = C1["n"], C1["steps"]
    u0 = torch.stack(spectral_field(n, seed=C1["seed"], device=f"cuda:{dev}")).contiguous()
    eta, tau = C1["etk_dns"], C1["tauk_dns"]
    fl = Flow(n, C1["nu"], C1["dt"], forcing=2, iseedf=C1["iseedf"], device=dev)
    fl.set_velocity(u0)
    del u0
    stream = torch.cuda.Stream(device=dev)
    fl.set_stream(stream)
    params = dict(nx=n, npart=C1["npart"], radius_um=C1["radius_um"], dt=C1["dt"], rnu=C1["nu"],
                  etk_dns=eta, tauk_dns=tau, device=dev)
    g = {}
    for p in ("fp64", "mixed"):
        g[p] = Partlib(ParticleParams(precision=p, **params))
        g[p].part_init()
        g[p].set_stream(stream)
    d = g["fp64"].scalars().d_coll
    sample_at = set(int(round(x)) for x in np.linspace(steps / C1["samples"], steps, C1["samples"]))
    samples = {p: [] for p in g}
    coll = {p: 0 for p in g}
    ms = {p: [] for p in g}
    t0 = time.perf_counter()
    for step in range(1, steps + 1):
        fl.step()
        vt = fl.velocity_tensors()
        for p, x in g.items():
            x.set_fields(*vt)
            if step not in sample_at:
                e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                e0.record(stream)
                rep, _ = x.particle_step()
                e1.record(stream)
                e1.synchronize()
                ms[p].append(e0.elapsed_time(e1))
                coll[p] += int(sum(rep.icc[:]))
                continue
            x.set_step(step, (step - 1) * C1["dt"])
            x.prepare_interp()
            for k in (1, 2, 3):
                x.interpolate(None, k)
            x.part_history_fvp()
            x.headlist(d)
            x.part_history_fdp()
            x.part_advance()
            x.complete_ypn()
            s = x.get_particles()
            before = x.histograms(written=False)["nirbin"].astype(np.int64)
            rep = x.collision_det()
            after = x.histograms(written=bool(rep.written))["nirbin"].astype(np.int64)
            coll[p] += int(sum(rep.icc[:]))
            samples[p].append({"step": step, "yp": s["yp"].copy(), "fvp": s["fvp"].copy(), "vp": s["vp"].copy(),
                               "dmove": s["dmove"].copy(), "icc": list(rep.icc[:]),
                               "pairs": sorted(map(tuple, x.pairs().tolist())),
                               "nirbin": after - before,
                               "candidates": int(rep.candidate_pairs)})
            x.update_part_position()
            x.periodic()
    wall = time.perf_counter() - t0
    for x in g.values():
        x.close()
    fl.close()
    return {"workload": "128^3 OU forcing (k <= sqrt 2), nu 0.0945, dt 1e-4, 2000 steps; 100,000 droplets "
                        "20/30 um (50/50)", "eta": eta, "tau_eta": tau, "d_coll": d,
            "samples": samples, "collisions": coll, "wall_s": wall,
            "particle_step_ms": {p: statistics.median(v) for p, v in ms.items()}}


def config4_bench(dev, torch, steps=4):
    """512^3 stochastic forcing, nu = 3e-4, 5,000,000 lognormal droplets (mean 25 um, sigma
    0.3, clipped to [10, 60] um) with HDI and coalescence (growth mode), the full mixed path:
    per-phase device times (flow transforms and kernels, interpolation, advance, cell list,
    collision, HDI, periodic/coalesce, overlap) and the algorithmic GB/s of the update and
    flow kernels."""
    import numpy as np
    from mpi_2d_domain_decomp_turb_particles_b200 import Partlib, ParticleParams
    from mpi_2d_domain_decomp_turb_particles_b200.bytes_model import (advance_bytes, flow_cross_bytes,
                                                                      flow_update_bytes, interp_bytes)
    from mpi_2d_domain_decomp_turb_particles_b200.flow import Flow
    from mpi_2d_domain_decomp_turb_particles_b200.synthetic import droplets, spectral_field
    n, npart = C4["n"], C4["npart"]
    field = spectral_field(n, seed=1234, device=f"cuda:{dev}")
    fl = Flow(n, C4["nu"], C4["dt"], forcing=2, iseedf=232300, device=dev)
    fl.set_velocity(torch.stack(field).contiguous())
    del field
    p = ParticleParams(nx=n, npart=npart, radius_um=[10.0, 25.0, 60.0], precision="mixed", device=dev,
                       new_particle=True, hdi_included=True, nonoverlap=True, hdi_trunc=50.0,
                       dt=C4["dt"], rnu=C4["nu"], etk_dns=C4["etk_dns"], tauk_dns=C4["tauk_dns"])
    g = Partlib(p)
    g.part_init()
    s = g.scalars()
    yp = droplets(npart, s.radius[1] / 25.0, lognormal=C4["lognormal"], seed=290710)
    lo, hi = (c * s.radius[1] / 25.0 for c in C4["clip_um"])
    yp[:, 6] = np.clip(yp[:, 6], lo, hi)
    g.set_particles(yp)
    stream = torch.cuda.Stream(device=dev)
    g.set_stream(stream)
    fl.set_stream(stream)
    g.set_step(40000, 0.0)             # growth mode: COALESCE on contact (turb.f90:591)
    fl.step(g)
    g.periodic()
    g.overlap_det()
    g.sync()
    fl.step(g)
    g.particle_step()
    torch.cuda.synchronize()
    fl.timing(True)
    flow_ms, step_ms, phases, iters = [], [], [], []
    for _ in range(steps):
        e = [torch.cuda.Event(enable_timing=True) for _ in range(3)]
        e[0].record(stream)
        fl.step(g)
        e[1].record(stream)
        _c, gm = g.particle_step()
        e[2].record(stream)
        torch.cuda.synchronize()
        flow_ms.append(e[0].elapsed_time(e[1]))
        step_ms.append(e[0].elapsed_time(e[2]))
        phases.append(g.phase_times())
        iters.append(gm.iterations)
    fparts = fl.timing(False)
    ph = np.median(np.array(phases), axis=0)
    nps = g.nps
    # the update kernels alone on the same droplets and field (the fused substep without
    # HDI), for the interpolation / advance split and their GB/s
    _, ukms, _, uims, uams = _time_update(g, stream, 5, 3, torch)
    g.close()
    fl.close()
    fft = fparts["fft_inverse"] + fparts["fft_forward"]
    return {"workload": "512^3 FP64 flow step (stochastic forcing, nu 3e-4) + 5M lognormal droplets (25 um, "
                        "sigma 0.3, [10, 60] um), HDI (50 radii) and coalescence, mixed",
            "step_ms": statistics.median(step_ms), "flow_step_ms": statistics.median(flow_ms),
            "breakdown_ms": {"fft": fft, "flow_cross_kernel": fparts["cross"], "flow_update_kernels": fparts["update"],
                             "interpolation": ph[7], "interp_to_history": ph[0], "advance": ph[6],
                             "cell_list": ph[1], "collision": ph[2], "hdi": ph[3], "periodic_coalesce": ph[4],
                             "overlap": ph[5]},
            "kernel_gbs": {"k_update (+forcing, finish)": _gbs(flow_update_bytes(n), fparts["update"]),
                           "k_cross_emit": _gbs(flow_cross_bytes(n), fparts["cross"]),
                           "k_interp_col": _gbs(interp_bytes("mixed", n, nps), uims),
                           "k_advance_fused": _gbs(advance_bytes("mixed", n, nps), uams)},
            "update_substep_kernels_ms": {"interp": uims, "advance": uams, "both": ukms},
            "droplets_after": nps, "gmres_iterations": iters,
            "note": "per-kernel times of k_coll_search, k_coll_eval, k_nei_walk, k_arn_solve, k_overlap: ncu launch list "
                    "of the same workload (bench.py --only config4)"}


def adjoint_bench(dev, torch):
    """128^3 field seeded as in the 64^3 case and run 300 forced FP64 steps (deterministic
    forcing), then frozen; 200,000 droplets of 25 um; 400 substeps checkpointed every 20.
    Forward and backward device time per substep for both precisions; central differences
    (h = 1e-6) of the FP64 loss on sampled entries of tau_p, x_0 and u against both
    adjoints; the mixed gradients' error against the FP64 adjoint."""
    import numpy as np
    from mpi_2d_domain_decomp_turb_particles_b200 import Partlib, ParticleParams
    from mpi_2d_domain_decomp_turb_particles_b200.adjoint import AdjointParams, DropletAdjoint
    n, npart = ADJ["n"], ADJ["np"]
    fl, u0 = _det_flow(n, ADJ["spin_nu"], ADJ["spin_dt"], ADJ["seed"], dev, torch)
    del u0
    for _ in range(ADJ["spinup"]):
        fl.step()
    u = torch.zeros((3, n, n, n + 2), dtype=torch.float64, device=f"cuda:{dev}")
    for c, t in enumerate(fl.velocity_tensors()):
        u[c, :, :, :n] = t
    fl.close()
    eps, eta, tau_k = _dissipation_scales(u.cpu().numpy(), ADJ["spin_nu"])
    phys = dict(dt=ADJ["dt"], rnu=ADJ["spin_nu"], etk_dns=eta, tauk_dns=tau_k)
    g = Partlib(ParticleParams(nx=n, npart=npart, radius_um=[ADJ["radius_um"]], precision="mixed",
                               device=dev, **phys))
    g.part_init()
    s = g.scalars()
    a_dns = s.radius[0]
    tau = s.tau_cloud_const2 * a_dns * a_dns
    grav = s.sv_const / s.tau_cloud_const2
    g.set_fields(*[u[c] for c in range(3)])
    stream = torch.cuda.Stream(device=dev)
    g.set_stream(stream)
    upd_ms, upd_kms, _, _, _ = _time_update(g, stream, 50, 5, torch)
    yp = g.get_particles()["yp"]
    g.close()
    x0 = np.ascontiguousarray(yp[:, :3])
    taus = np.full(npart, tau)
    rad = np.full(npart, a_dns)
    out, grads, probs = {}, {}, {}
    for prec in ("mixed", "fp64"):
        p = AdjointParams(n=n, nsteps=ADJ["nsteps"], dt=ADJ["dt"], gravity=grav, precision=prec,
                          checkpoint_every=ADJ["checkpoint_every"], pair_factor=ADJ["pair_factor"], device=dev)
        a = DropletAdjoint(p, npart)
        a.set_field(u)
        tx = torch.tensor(x0, device=f"cuda:{dev}")
        tt = torch.tensor(taus, device=f"cuda:{dev}")
        tr = torch.tensor(rad, device=f"cuda:{dev}")
        a.set_droplets(tx, tt, tr)
        dx0 = torch.zeros((npart, 3), dtype=torch.float64, device=f"cuda:{dev}")
        dtau = torch.zeros(npart, dtype=torch.float64, device=f"cuda:{dev}")
        du = torch.zeros_like(u)
        torch.cuda.synchronize()
        for _ in range(2):   # the second pair is timed
            loss, npairs = a.forward()
            a.backward(dx0, dtau, du)
        fms, bms = a.timing()
        steps = ADJ["nsteps"]
        out[prec] = {"forward_ms_per_step": fms / steps, "backward_ms_per_step": bms / steps,
                     "adjoint_over_forward": bms / fms, "loss": loss, "pairs": npairs}
        grads[prec] = (dx0.cpu().numpy(), dtau.cpu().numpy(), du.cpu().numpy())
        probs[prec] = a
    # central differences of the FP64 loss
    a64 = probs["fp64"]
    h = ADJ["fd_h"]
    rng = np.random.default_rng(11)
    k = ADJ["fd_entries"]
    u_host = u.cpu().numpy()

    def loss_at(u_=None, x_=None, t_=None):
        if u_ is not None:
            a64.set_field(u_)
        a64.set_droplets(x_ if x_ is not None else x0, t_ if t_ is not None else taus, rad)
        val = a64.forward()[0]
        if u_ is not None:
            a64.set_field(u)
        return val

    g64, gmx = grads["fp64"], grads["mixed"]
    fd = {"tau": [], "x0": [], "u": []}
    for i in rng.choice(npart, k, replace=False):
        tp_, tm = taus.copy(), taus.copy()
        tp_[i] += h; tm[i] -= h
        fd["tau"].append(((int(i),), (loss_at(t_=tp_) - loss_at(t_=tm)) / (2 * h), g64[1][i], gmx[1][i]))
    for i in rng.choice(npart, k, replace=False):
        c = int(rng.integers(3))
        xp, xm = x0.copy(), x0.copy()
        xp[i, c] += h; xm[i, c] -= h
        fd["x0"].append(((int(i), c), (loss_at(x_=xp) - loss_at(x_=xm)) / (2 * h), g64[0][i, c], gmx[0][i, c]))
    du64 = g64[2][:, :, :, :n]
    flat = np.argsort(np.abs(du64).ravel())
    picks = list(flat[-(k // 2):]) + list(rng.choice(flat[-du64.size // 4:], k - k // 2, replace=False))
    for q in picks:
        idx = np.unravel_index(q, du64.shape)
        up, um = u_host.copy(), u_host.copy()
        up[idx] += h; um[idx] -= h
        fd["u"].append((tuple(int(v) for v in idx), (loss_at(u_=up) - loss_at(u_=um)) / (2 * h),
                        g64[2][idx], gmx[2][idx]))
    for a in probs.values():
        a.close()

    def fd_err(rows, j, scale):
        return max(abs(r[j] - r[1]) / max(abs(r[1]), 1e-3 * scale) for r in rows)

    fdrep = {}
    for nm, j in (("tau", 1), ("x0", 0), ("u", 2)):
        scale = float(np.abs(g64[j]).max())
        fdrep[nm] = {"entries": len(fd[nm]), "fp64_max_rel": fd_err(fd[nm], 2, scale),
                     "mixed_max_rel": fd_err(fd[nm], 3, scale),
                     "rows": [[list(r[0]), r[1], float(r[2]), float(r[3])] for r in fd[nm][:3]]}

    def rel(a_, b_):
        return float(np.abs(a_ - b_).max() / max(np.abs(b_).max(), 1e-300))

    return {"workload": "128^3 field: seeded spectrum + 300 FP64 steps of deterministic forcing (nu 0.0025, "
                        "dt 1e-3), frozen; 200,000 droplets of 25 um, 400 substeps (dt 5e-4), checkpoint every "
                        "20; loss = mean w_r of pairs within 2(a_i+a_j) + mean |x_T - x_0|^2",
            "spinup_epsilon": eps, "mixed": out["mixed"], "fp64": out["fp64"],
            "update_step_ms_same_config": upd_ms, "update_kernels_ms_same_config": upd_kms,
            "adjoint_over_update_step": out["mixed"]["backward_ms_per_step"] / upd_ms,
            "finite_differences": {"h": h, "denominator": "max(|fd|, 1e-3 max|grad|)", **fdrep},
            "mixed_vs_fp64_gradient_rel": {"x0": rel(gmx[0], g64[0]), "tau": rel(gmx[1], g64[1]),
                                           "u": rel(gmx[2], g64[2])},
            "loss_rel_mixed_vs_fp64": abs(out["mixed"]["loss"] - out["fp64"]["loss"]) / abs(out["fp64"]["loss"])}


# ---------------------------------------------------------------------------------------
# CPU leg: the FP64 oracle timed on the host's cores, and the checker of the GPU legs
# ---------------------------------------------------------------------------------------
def _oracle_mod():
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as orc
    orc.build()
    return orc


def _oracle_sample(npart, steps, field=None, min_seconds=0.0, warmup=1):
    """Oracle update steps (FP64 CPU restatement) on the headline workload's first `npart`
    droplets: returns (updates/s, threads, s/step)."""
    import numpy as np
    from mpi_2d_domain_decomp_turb_particles_b200.synthetic import droplets, spectral_field
    orc = _oracle_mod()
    o = orc.Oracle(nx=N_GRID, ny=N_GRID, nz=N_GRID, npart=npart, radius_um=SETS_UM, **PHYS)
    o.part_init()
    scale = o.yp[0, 6] / SETS_UM[0] if o.nps else 1.0
    yp = droplets(npart, scale, radius_um=(10.0, 40.0), seed=290710)
    o.nps = npart
    o.yp[:npart] = yp
    if field is None:
        field = [np.ascontiguousarray(t.numpy()) for t in spectral_field(N_GRID, seed=1234, device="cpu")]
    for _ in range(max(1, warmup)):
        o.update_step(*field)
    t = time.perf_counter()
    done = 0
    while done < steps or (time.perf_counter() - t) < min_seconds:
        o.update_step(*field)
        done += 1
        if done >= 200:
            break
    dt = (time.perf_counter() - t) / done
    return npart / dt, orc.num_threads(), dt


def _cpu_model():
    try:
        with open("/proc/cpuinfo") as f:
            for line in f:
                if line.startswith("model name"):
                    return line.split(":", 1)[1].strip()
    except OSError:
        pass
    return None


def _cpu_flow_step(n=N_GRID):
    """One FP64 flow step of the numpy/scipy restatement (scipy.fft, all cores)."""
    import numpy as np
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    from flow_oracle import FlowOracle
    rng = np.random.default_rng(3)
    f = FlowOracle(n, PHYS["rnu"], PHYS["dt"], forcing=1, force=(0.3, 0.2), workers=-1)
    f.set_velocity(rng.standard_normal((3, n, n, n)))
    f.step()
    t = time.perf_counter()
    f.step()
    return time.perf_counter() - t


def _oracle_errors(orc, rec, field):
    """The oracle on the errors leg's inputs: relative error of each floating-point output
    of both GPU paths against it, and whether the FP64 path and the pair lists are exact."""
    import numpy as np
    from mpi_2d_domain_decomp_turb_particles_b200 import ParticleParams
    yp0 = rec["yp0"]
    n = yp0.shape[0]
    p = ParticleParams(nx=N_GRID, npart=n, radius_um=SETS_UM, new_particle=True, **PHYS)
    o = orc.Oracle(**p.oracle_kwargs())
    o.part_init()
    o.nps = n
    o.yp[:n] = yp0
    o.prepare_interp()
    for k in range(3):
        o.interpolate(field[k], k + 1)
    vo = o.vp[:n].copy()
    ref = {"icc": [], "wr": [], "pairs": []}
    hist = _Hist()
    t = time.perf_counter()
    for _ in range(rec["steps"]):
        r = o.particle_step(*field)
        ref["icc"].append(r["icc"].tolist())
        hist.oracle_step(o)
        c = r["contacts"]
        ref["wr"].append(np.array([x[3][11] for x in c]) if len(c) else np.zeros(0))
        ref["pairs"].append(sorted((int(x[0]), int(x[2]), int(x[3]), int(x[4])) for x in r["pairs"]))
    wall = time.perf_counter() - t
    hist.oracle_end(o)
    ypo = o.yp[:o.nps].copy()
    urms = float(np.sqrt(np.mean(vo ** 2)))
    radius = rec["radius_sets"]

    def settle(yp):
        sidx = np.argmin(np.abs(yp[:, 6][:, None] - radius[None, :]), axis=1)
        return np.array([yp[sidx == k, 3].mean() for k in range(len(radius))])

    so = settle(ypo)
    nir_o, wr_o = hist.nir, hist.wr
    wc_o = np.concatenate(ref["wr"])
    out = {"reference": "FP64 CPU oracle (restatement of partlib.f90) on the same 1M droplets and 256^3 field",
           "steps": rec["steps"], "oracle_wall_s": wall}
    for prec in ("mixed", "fp64"):
        r = rec[prec]
        v = r["vp"]
        nir, wr = r["nirbin"], r["wrbin"]
        wc = np.concatenate(r["wr"])
        nz = nir_o > 0
        mean_o = np.where(nz, wr_o / np.maximum(nir_o, 1), 0.0)
        mean_g = np.where(nir > 0, wr / np.maximum(nir, 1), 0.0)
        coll_g, coll_o = int(np.sum(r["icc"])), int(np.sum(ref["icc"]))
        out[prec] = {
            "interpolated_velocity": {"rel_l2": float(np.linalg.norm(v - vo) / np.linalg.norm(vo)),
                                      "max_abs_over_urms": float(np.abs(v - vo).max() / urms),
                                      "bit_identical": bool(np.array_equal(v, vo))},
            "settling_velocity_rel_per_set": (np.abs(settle(r["yp"]) - so) / np.abs(so)).tolist(),
            "rdf_bins": {"rel_l2": float(np.linalg.norm(nir - nir_o) / max(np.linalg.norm(nir_o), 1e-300)),
                         "pairs_counted": int(nir_o.sum()), "identical": bool(np.array_equal(nir, nir_o))},
            "wr_per_bin_mean": {"max_rel": float(np.max(np.abs(mean_g[nz] - mean_o[nz]) /
                                                        np.maximum(np.abs(mean_o[nz]), 1e-300))) if nz.any() else None,
                                "bins_used": int(nz.sum())},
            "wr_at_contact_records": {"rel": float(abs(wc.mean() - wc_o.mean()) / abs(wc_o.mean()))
                                      if wc.size and wc_o.size and wc.size == wc_o.size else None,
                                      "records": [int(wc.size), int(wc_o.size)]},
            "collision_kernel": {"collisions": coll_g, "collisions_oracle": coll_o,
                                 "rel": float(abs(coll_g - coll_o) / coll_o) if coll_o else None},
            "pair_lists_identical_per_step": [a == b for a, b in zip(r["pairs"], ref["pairs"])],
        }
    out["fp64"]["state_bit_identical_after_steps"] = bool(np.array_equal(rec["fp64"]["yp"], ypo))
    out["settling_velocity_sets_um"] = SETS_UM
    return out


def _oracle_config0(orc, rec, dev):
    """The oracle through the same 500 flow fields (the deterministic device flow run
    again; each field's checksum must match the GPU leg's) with the FP64 droplet path's
    parameters: RDF at contact, w_r at contact, collision count."""
    import numpy as np
    import torch
    from mpi_2d_domain_decomp_turb_particles_b200 import ParticleParams
    n = C0["n"]
    p = ParticleParams(nx=n, npart=C0["npart"], radius_um=[C0["radius_um"]], dt=C0["dt"], rnu=C0["nu"],
                       etk_dns=rec["eta"], tauk_dns=rec["tau_eta"], ediss_cloud=C0["ediss_cloud"],
                       gravity=C0["gravity"])
    o = orc.Oracle(**p.oracle_kwargs())
    o.part_init()
    o.seti("init_velocity", 1)
    fl, u0 = _det_flow(n, C0["nu"], C0["dt"], C0["seed"], dev, torch)
    del u0
    hist = _Hist()
    coll = 0
    same_fields = True
    t = time.perf_counter()
    for k in range(C0["steps"]):
        fl.step()
        vt = fl.velocity_tensors()
        same_fields &= _field_sum(vt) == rec["field_sums"][k]
        f = [np.ascontiguousarray(x.cpu().numpy()) for x in vt]
        r = o.particle_step(*f)
        hist.oracle_step(o)
        coll += int(r["icc"].sum())
    wall = time.perf_counter() - t
    hist.oracle_end(o)
    fl.close()
    a = o.yp[0, 6] if o.nps else 0.0
    expect = _rdf_expected(C0["npart"], 2 * a, C0["steps"])
    oracle = _rdf_summary(hist.nir[:, 0, 0], hist.wr[:, 0, 0], expect)
    nir = oracle.pop("nirbin")
    oracle.update(collisions=coll, wall_s=wall)
    res = {k: v for k, v in rec.items() if k not in ("field_sums",)}

    def rel(x, y):
        return abs(x - y) / abs(y) if x is not None and y else None

    for prec in ("fp64", "mixed"):
        r = dict(rec[prec])
        nb = r.pop("nirbin")
        r["nirbin_identical_to_oracle"] = bool(np.array_equal(nb, nir))
        for key in ("rdf_contact", "wr_contact", "rdf_near_contact", "wr_near_contact"):
            r[key + "_rel"] = rel(r[key], oracle[key])
        res[prec] = r
    res["oracle"] = oracle
    res["same_fields_as_gpu_leg"] = bool(same_fields)
    return res


def _oracle_config1(orc, rec):
    """COLLISION_DET of the oracle on each sampled state of each path (identical inputs):
    pair lists, collision counts and RDF counts compared."""
    import numpy as np
    from mpi_2d_domain_decomp_turb_particles_b200 import ParticleParams
    p = ParticleParams(nx=C1["n"], npart=C1["npart"], radius_um=C1["radius_um"], dt=C1["dt"], rnu=C1["nu"],
                       etk_dns=rec["eta"], tauk_dns=rec["tau_eta"])
    o = orc.Oracle(**p.oracle_kwargs())
    o.part_init()
    checks = {}
    t = time.perf_counter()
    for prec, samples in rec["samples"].items():
        rows = []
        for s in samples:
            m = s["yp"].shape[0]
            o.nps = m
            o.yp[:m] = s["yp"]
            o.fvp[:m] = s["fvp"]
            o.dmove[:m] = s["dmove"]
            o.vp[:m] = s["vp"]
            o.seti("istep", s["step"])
            o.headlist(rec["d_coll"])
            o.complete_ypn()
            before = o.hist("nirbin").astype(np.int64)
            o.collision_det()
            after = o.hist("out_nirbin" if o.geti("written") else "nirbin").astype(np.int64)
            op = sorted((int(r[0]), int(r[2]), int(r[3]), int(r[4])) for r in o.pairs())
            rows.append({"step": s["step"], "pairs": len(op), "rdf_pairs": int((after - before).sum()),
                         "pairs_identical": s["pairs"] == op,
                         "icc_identical": s["icc"] == o.arr("icc", np.int32).tolist(),
                         "nirbin_identical": bool(np.array_equal(s["nirbin"], after - before)),
                         "candidates_identical": s["candidates"] == o.getl("candidate_pairs")})
        checks[prec] = {"sampled_steps": [r["step"] for r in rows],
                        "all_pairs_identical": all(r["pairs_identical"] for r in rows),
                        "all_counts_identical": all(r["icc_identical"] and r["nirbin_identical"] and
                                                    r["candidates_identical"] for r in rows),
                        "collision_pairs_total": sum(r["pairs"] for r in rows),
                        "rdf_pairs_total": sum(r["rdf_pairs"] for r in rows)}
    res = {k: v for k, v in rec.items() if k != "samples"}
    res["oracle_detection_on_identical_inputs"] = checks
    res["oracle_wall_s"] = time.perf_counter() - t
    return res


def cpu_baseline(rec=None, field=None, dev=0):
    """The CPU leg: the oracle timed on this host's cores on a bounded sample of the
    headline workload (same field and droplets), then the oracle as the checker of the
    recorded GPU legs.  Returns the cpu_baseline object (plus the checker's results under
    "errors", "config0", "config1", which the caller moves to their own keys)."""
    import numpy as np
    orc = _oracle_mod()
    rec = rec or {}
    if field is None:
        from mpi_2d_domain_decomp_turb_particles_b200.synthetic import spectral_field
        field = [np.ascontiguousarray(t.numpy()) for t in spectral_field(N_GRID, seed=1234, device="cpu")]
    else:
        field = [np.ascontiguousarray(f) for f in field]
    npart = 200_000
    v, th, dt = _oracle_sample(npart, 3, field, min_seconds=10.0)
    orc.set_num_threads(1)
    n1 = 20_000
    v1, _, dt1 = _oracle_sample(n1, 3, field, min_seconds=4.0)
    orc.set_num_threads(th)
    flow_s = _cpu_flow_step()
    out = {"value": v, "unit": "particle-updates/s", "cores": th, "kind": "port",
           "sample": f"{npart} droplets drawn as the headline's (radii U[10, 40] um) in the same seeded 256^3 FP64 "
                     f"field, >= 10 s of update steps "
                     f"(interpolation + history + advance + position), OpenMP over droplets; {dt:.3f} s/step",
           "cpu_model": _cpu_model(), "one_core_value": v1,
           "one_core_sample": f"{n1} droplets, 1 thread, {dt1:.3f} s/step",
           "flow_step_s_256": flow_s,
           "flow_sample": f"one 256^3 FP64 flow step of the numpy restatement with scipy.fft on {os.cpu_count()} "
                          f"workers"}
    if "errors" in rec:
        out["errors"] = _oracle_errors(orc, rec["errors"], field)
    if "config0" in rec:
        out["config0"] = _oracle_config0(orc, rec["config0"], dev)
    if "config1" in rec:
        out["config1"] = _oracle_config1(orc, rec["config1"])
    return out


# ---------------------------------------------------------------------------------------
def run_only(args):
    """One workload alone, for profilers (ncu launch lists and kernel captures): prints
    a short JSON line with its device time; no baselines, no extra workloads."""
    import torch
    torch.cuda.set_device(0)
    from mpi_2d_domain_decomp_turb_particles_b200.synthetic import spectral_field
    out = {"only": args.only}
    if args.only in ("update", "update-fp64"):
        field = spectral_field(N_GRID, seed=1234, device="cuda:0")
        g = _make("mixed" if args.only == "update" else "fp64", 0)
        stream = torch.cuda.Stream()
        g.set_stream(stream)
        g.set_fields(*field)
        g.sync()
        ms, kms, launches, ims, ams = _time_update(g, stream, args.steps, args.warmup, torch)
        out.update(ms_per_step=ms, kernel_ms=kms, launches=launches, interp_ms=ims, advance_ms=ams)
        g.close()
    elif args.only == "step":
        # the full mixed particle substep without HDI (cell list, collision detection and
        # statistics) on the headline workload
        field = spectral_field(N_GRID, seed=1234, device="cuda:0")
        g = _make("mixed", 0)
        stream = torch.cuda.Stream()
        g.set_stream(stream)
        g.set_fields(*field)
        g.sync()
        for _ in range(args.warmup):
            g.particle_step()
        ts, ph = [], []
        for _ in range(args.steps):
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            rep, _ = g.particle_step()
            e1.record(stream)
            torch.cuda.synchronize()
            ts.append(e0.elapsed_time(e1))
            ph.append(g.phase_times().tolist())
        out.update(step_ms=statistics.median(ts), phase_ms=ph[-1], candidates=int(rep.candidate_pairs))
        g.close()
    elif args.only == "adjoint":
        out.update(adjoint_bench(0, torch))
    elif args.only == "full":
        field = spectral_field(N_GRID, seed=1234, device="cuda:0")
        out.update(full_step_bench(0, torch, field))
    elif args.only == "config4":
        out.update(config4_bench(0, torch))
    elif args.only == "configs":
        import numpy as np
        r0, r1 = config0_gpu(0, torch), config1_gpu(0, torch)
        r0.pop("field_sums")
        for p in ("fp64", "mixed"):
            r0[p].pop("nirbin")
        r1.pop("samples")
        out.update(config0=r0, config1=r1)
    print(json.dumps(out, default=float), flush=True)


def run_reference(args):
    ws, rank, local = _dist()
    if rank != 0:
        return
    npart = args.ref_sample
    v, th, dt = _oracle_sample(npart, args.steps, warmup=args.warmup)
    line = {
        "metric": "particle-updates/s (256^3, 1M droplets, mixed precision)", "impl": "reference",
        "value": v, "unit": "particle-updates/s", "n_gpus": ws, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": dt * 1e3 * N_PART / npart, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic", "config": CONFIG,
        "cpu_baseline": {"value": v, "unit": "particle-updates/s", "cores": th, "kind": "port",
                         "sample": f"{npart} droplets per step drawn as the headline's, in the same seeded 256^3 field "
                                   f"(FP64 CPU restatement of partlib.f90; the Fortran/MPI reference cannot "
                                   f"be built here)"},
        "e2e": {"value": v, "unit": "particle-updates/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=1000)
    ap.add_argument("--warmup", type=int, default=10)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--no-adjoint", action="store_true", help="skip the adjoint workload")
    ap.add_argument("--no-full", action="store_true", help="skip the flow + HDI full-step workload")
    ap.add_argument("--no-config4", action="store_true", help="skip the 512^3 / 5M-droplet workload")
    ap.add_argument("--no-configs", action="store_true", help="skip the 64^3 and 128^3 workloads")
    ap.add_argument("--ref-sample", type=int, default=200_000,
                    help="droplets per step of the reference arm's CPU sample")
    ap.add_argument("--only", choices=["update", "update-fp64", "step", "adjoint", "full", "config4", "configs"],
                    help="run one workload alone (for profilers)")
    args = ap.parse_args()
    args.warmup = max(3, args.warmup)
    if args.impl == "reference":
        run_reference(args)
    elif args.only:
        run_only(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
