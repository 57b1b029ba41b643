"""Benchmark of the droplet update path (particle-updates/s) on B200.

Workload (N = 1): the headline configuration's shape -- a 256^3 periodic field and
1,000,000 droplets with radii uniform in [10, 40] um -- with the mixed-precision path as
the measured value and the FP64 path beside it.  One "step" is one droplet substep of the
update path: interpolation of the three velocity components, history, drag advance,
position update, periodic wrap and the PERIODIC reorder (plus the amortised spatial
re-sort of the device order).  Inputs (field, droplet state) are resident in HBM when the
timed region starts and are larger than L2 (field 218 MB FP32 / 441 MB FP64, droplet
state ~0.2 GB), so no L2 flush is needed.  N > 1 runs independent replicas, one per GPU
(the path does not shard on one node; weak scaling).

``--impl reference`` times the CPU restatement of the reference's path (the reference
itself cannot be built here) on this host's cores on a bounded sample of droplets.
"""
from __future__ import annotations

import argparse
import json
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


def _make(precision, dev, npart=N_PART, n=N_GRID, hdi=False):
    import numpy as np
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
    kms, nk, launches = g.timing(reset=True)
    return ms / steps, kms, launches


def run_ours(args):
    import torch
    import torch.distributed as dist
    from mpi_2d_domain_decomp_turb_particles_b200.bytes_model import update_bytes

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
    ms_step, kernel_ms, launches = _time_update(g, stream, args.steps, args.warmup, torch)
    clocks = _clock_summary(clk)
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
    import numpy as np
    host = [f.cpu().pin_memory() for f in field]
    e2e_steps = max(1, min(args.steps, 5))
    for _ in range(2):
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
    del g

    # ---- FP64 path, same workload ----
    g64 = _make("fp64", dev)
    g64.set_stream(stream)
    g64.set_fields(*field)
    g64.sync()
    ms64, kms64, _ = _time_update(g64, stream, max(3, args.steps // 2), args.warmup, torch)
    g64.close()
    (ms64,) = max_over_ranks([ms64], ws, device=f"cuda:{dev}")
    value64 = replica_value(ws, N_PART, ms64)

    errs = errors_bench(dev, torch, field)
    adj = adjoint_bench(dev, torch) if not args.no_adjoint else None
    full = full_step_bench(dev, torch, field) if not args.no_full else None
    del field
    torch.cuda.empty_cache()
    c4 = None
    if not args.no_config4:
        try:
            c4 = config4_bench(dev, torch)
        except Exception as ex:   # reported, not fatal: the headline numbers stand alone
            c4 = {"error": f"{type(ex).__name__}: {ex}"}

    if rank == 0:
        peak, kind = _peaks()
        alg = update_bytes("mixed", N_GRID, N_PART)
        achieved = alg / (kernel_ms * 1e-3) / 1e9
        traffic = _profile_traffic()
        line = {
            "metric": "particle-updates/s (256^3, 1M droplets, mixed precision)",
            "value": value, "unit": "particle-updates/s", "n_gpus": ws, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms_step, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32 (positions f64)", "data": "synthetic (seeded spectrum field, uniform droplets)",
            "config": CONFIG,
            "fp64_value": value64, "fp64_ms_per_step": ms64, "mixed_over_fp64": value / value64,
            "full_step_ms": full_ms, "collision_ms": coll_ms,
            "collision_candidate_pairs_per_s": cand / (coll_ms * 1e-3) if coll_ms > 0 else None,
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": achieved / peak, "traffic": traffic, "peak_kind": f"{kind} (burst copy)",
                         "kernel": "k_interp + k_advance_fused, per update step",
                         "algorithmic_bytes": alg, "kernel_ms": kernel_ms},
            "e2e": {"value": N_PART / (e2e_ms * 1e-3), "unit": "particle-updates/s",
                    "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h,
                    "path": "dl_set_field (host FP64 field, pinned) + dl_update_step + dl_mean_vel"},
            "errors_vs_fp64": errs,
            "full_step": full,
            "config4": c4,
            "adjoint": adj,
            "gpu_launches": int(launches),
            "clocks": clocks,
            "cpu_baseline": cpu_baseline(),
        }
        print(json.dumps(line), flush=True)
    if ws > 1:
        dist.barrier()
        dist.destroy_process_group()


def full_step_bench(dev, torch, field):
    """The whole time step of the headline configuration: the device flow step (256^3 FP64
    pseudo-spectral, stochastic forcing) and the droplet substep with hydrodynamic
    interaction (1M droplets, radii U[10, 40] um, mixed precision), device time per step."""
    from mpi_2d_domain_decomp_turb_particles_b200.flow import Flow
    fl = Flow(N_GRID, PHYS["rnu"], PHYS["dt"], forcing=2, iseedf=232300, device=dev)
    u = torch.stack(field).contiguous()
    fl.set_velocity(u)
    stream = torch.cuda.Stream(device=dev)
    fl.set_stream(stream)
    for _ in range(3):
        fl.step()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    nf = 10
    e0.record(stream)
    for _ in range(nf):
        fl.step()
    e1.record(stream)
    torch.cuda.synchronize()
    flow_ms = e0.elapsed_time(e1) / nf
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
    ts, iters = [], []
    for _ in range(5):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        fl.step(g)
        _c, gm = g.particle_step()
        e1.record(stream)
        torch.cuda.synchronize()
        ts.append(e0.elapsed_time(e1))
        iters.append(gm.iterations)
    ph = g.phase_times()
    g.close()
    fl.close()
    return {"workload": "256^3 FP64 flow step (stochastic forcing) + 1M-droplet substep with HDI (50 radii), mixed",
            "flow_step_ms": flow_ms, "step_ms": statistics.median(ts),
            "particle_phase_ms": {"interp_advance": ph[0], "cell_list": ph[1], "collision": ph[2], "hdi": ph[3],
                                  "periodic_relocate": ph[4], "overlap": ph[5]},
            "gmres_iterations": iters}


def errors_bench(dev, torch, field, steps=10):
    """Relative error of each floating-point output of the mixed path against the FP64
    path (bit-identical to the FP64 oracle on identical inputs) on the headline workload:
    interpolated velocity at identical positions, then over `steps` full particle steps
    (collision detection and statistics on) the settling velocity (set means of yp(4)),
    the RDF bins, w_r at contact and the collision kernel (collision counts)."""
    import numpy as np
    g = {p: _make(p, dev) for p in ("mixed", "fp64")}
    for x in g.values():
        x.set_fields(*field)
        x.prepare_interp()
        for k in (1, 2, 3):
            x.interpolate(None, k)
    vm, v64 = g["mixed"].get_particles()["vp"], g["fp64"].get_particles()["vp"]
    urms = float(np.sqrt(np.mean(v64 ** 2)))
    out = {"interpolated_velocity": {"rel_l2": float(np.linalg.norm(vm - v64) / np.linalg.norm(v64)),
                                     "max_abs_over_urms": float(np.abs(vm - v64).max() / urms)}}
    acc = {p: {"icc": np.zeros(3), "wr": [], "nir": None} for p in g}
    for p, x in g.items():
        for _ in range(steps):
            rep, _gm = x.particle_step()
            acc[p]["icc"] += np.array(rep.icc[:])
            if rep.ncontact:
                acc[p]["wr"].append(x.contacts()[1][:, 11])
            if rep.written:
                acc[p]["nir"] = x.histograms(written=True)["nirbin"].astype(np.float64)
    radius = np.array(g["fp64"].scalars().radius[:len(SETS_UM)])
    settle = {}
    for p, x in g.items():
        yp = x.get_particles()["yp"]
        sidx = np.argmin(np.abs(yp[:, 6][:, None] - radius[None, :]), axis=1)
        settle[p] = np.array([yp[sidx == k, 3].mean() for k in range(len(SETS_UM))])
    out["settling_velocity"] = {"rel_per_set": (np.abs(settle["mixed"] - settle["fp64"]) /
                                                np.abs(settle["fp64"])).tolist(),
                                "sets_um": SETS_UM}
    nm, n64 = acc["mixed"]["nir"], acc["fp64"]["nir"]
    out["rdf_bins"] = {"rel_l2": float(np.linalg.norm(nm - n64) / max(np.linalg.norm(n64), 1e-300)),
                       "pairs_counted": int(n64.sum())}
    wm = np.concatenate(acc["mixed"]["wr"]) if acc["mixed"]["wr"] else np.zeros(0)
    w64 = np.concatenate(acc["fp64"]["wr"]) if acc["fp64"]["wr"] else np.zeros(0)
    out["wr_at_contact"] = {"mean_mixed": float(wm.mean()) if wm.size else None,
                            "mean_fp64": float(w64.mean()) if w64.size else None,
                            "rel": float(abs(wm.mean() - w64.mean()) / abs(w64.mean())) if wm.size and w64.size else None,
                            "records": [int(wm.size), int(w64.size)]}
    cm, c64 = acc["mixed"]["icc"].sum(), acc["fp64"]["icc"].sum()
    out["collision_kernel"] = {"collisions_mixed": int(cm), "collisions_fp64": int(c64),
                               "rel": float(abs(cm - c64) / c64) if c64 else None}
    out["steps"] = steps
    out["reference"] = "FP64 GPU path (bit-identical to the FP64 oracle on identical inputs)"
    for x in g.values():
        x.close()
    return out


C4 = dict(n=512, npart=5_000_000, nu=3e-4, dt=5e-4, etk_dns=0.00484, tauk_dns=0.078, lognormal=(25.0, 0.3),
          clip_um=(10.0, 60.0))


def config4_bench(dev, torch, steps=4):
    """512^3 stochastic forcing, nu = 3e-4, 5,000,000 lognormal droplets (mean 25 um, sigma
    0.3, clipped to [10, 60] um) with HDI and coalescence (growth mode), the full mixed path:
    per-phase device times and the update phase's algorithmic HBM GB/s."""
    import numpy as np
    from mpi_2d_domain_decomp_turb_particles_b200 import Partlib, ParticleParams
    from mpi_2d_domain_decomp_turb_particles_b200.bytes_model import update_bytes
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
    ph = np.median(np.array(phases), axis=0)
    nps = g.nps
    upd_gbs = update_bytes("mixed", n, nps) / (ph[0] * 1e-3) / 1e9 if ph[0] > 0 else None
    g.close()
    fl.close()
    return {"workload": "512^3 FP64 flow step (stochastic forcing, nu 3e-4) + 5M lognormal droplets (25 um, "
                        "sigma 0.3, [10, 60] um), HDI (50 radii) and coalescence, mixed",
            "step_ms": statistics.median(step_ms), "flow_step_ms": statistics.median(flow_ms),
            "particle_phase_ms": {"interp_advance": ph[0], "cell_list": ph[1], "collision": ph[2], "hdi": ph[3],
                                  "periodic_coalesce": ph[4], "overlap": ph[5]},
            "update_phase_algorithmic_gbs": upd_gbs, "droplets_after": nps, "gmres_iterations": iters}


ADJ = dict(n=128, np=200_000, radius_um=25.0, nsteps=400, checkpoint_every=20, dt=5e-4,
           etk_dns=0.0158, tauk_dns=0.156, pair_factor=2.0)


def adjoint_bench(dev, torch):
    """Adjoint workload (128^3 frozen field, 200,000 droplets of 25 um, 400 substeps,
    checkpoint every 20): device time of the forward pass and of the backward pass
    (recompute + reverse sweep), per substep, beside the production update step on the
    same field and droplets."""
    import numpy as np
    from mpi_2d_domain_decomp_turb_particles_b200 import Partlib, ParticleParams
    from mpi_2d_domain_decomp_turb_particles_b200.adjoint import AdjointParams, DropletAdjoint
    from mpi_2d_domain_decomp_turb_particles_b200.synthetic import spectral_field
    n, npart = ADJ["n"], ADJ["np"]
    phys = dict(dt=ADJ["dt"], rnu=PHYS["rnu"], etk_dns=ADJ["etk_dns"], tauk_dns=ADJ["tauk_dns"])
    g = Partlib(ParticleParams(nx=n, npart=npart, radius_um=[ADJ["radius_um"]], precision="mixed",
                               device=dev, **phys))
    g.part_init()
    s = g.scalars()
    a_dns = s.radius[0]
    tau = s.tau_cloud_const2 * a_dns * a_dns
    grav = s.sv_const / s.tau_cloud_const2
    field = spectral_field(n, seed=1234, device=f"cuda:{dev}")
    g.set_fields(*field)
    stream = torch.cuda.Stream(device=dev)
    g.set_stream(stream)
    upd_ms, upd_kms, _ = _time_update(g, stream, 50, 5, torch)
    yp = g.get_particles()["yp"]
    g.close()
    x0 = torch.tensor(np.ascontiguousarray(yp[:, :3]), device=f"cuda:{dev}")
    taus = torch.full((npart,), tau, dtype=torch.float64, device=f"cuda:{dev}")
    rad = torch.full((npart,), a_dns, dtype=torch.float64, device=f"cuda:{dev}")
    u = torch.stack(field).contiguous()
    out = {}
    for prec in ("mixed", "fp64"):
        p = AdjointParams(n=n, nsteps=ADJ["nsteps"], dt=ADJ["dt"], gravity=grav, precision=prec,
                          checkpoint_every=ADJ["checkpoint_every"], pair_factor=ADJ["pair_factor"], device=dev)
        a = DropletAdjoint(p, npart)
        a.set_field(u)
        a.set_droplets(x0, taus, rad)
        dx0 = torch.zeros((npart, 3), dtype=torch.float64, device=f"cuda:{dev}")
        dtau = torch.zeros(npart, dtype=torch.float64, device=f"cuda:{dev}")
        du = torch.zeros_like(u)
        torch.cuda.synchronize()
        for _ in range(2):   # the second pair is timed
            loss, npairs = a.forward()
            a.backward(dx0, dtau, du)
        fms, bms = a.timing()
        a.close()
        steps = ADJ["nsteps"]
        out[prec] = {"forward_ms_per_step": fms / steps, "backward_ms_per_step": bms / steps,
                     "adjoint_over_forward": bms / fms, "loss": loss, "pairs": npairs}
    return {"workload": "128^3 frozen synthetic field, 200,000 droplets of 25 um, 400 substeps, "
                        "checkpoint every 20; loss = mean w_r of pairs within 2(a_i+a_j) + mean |x_T - x_0|^2",
            "mixed": out["mixed"], "fp64": out["fp64"],
            "update_step_ms_same_config": upd_ms, "update_kernels_ms_same_config": upd_kms,
            "adjoint_over_update_step": out["mixed"]["backward_ms_per_step"] / upd_ms}


def _oracle_sample(npart, n, steps, min_seconds=0.0):
    """Oracle (CPU restatement) update steps on a sample: returns (updates/s, threads)."""
    import numpy as np
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as orc
    orc.build()
    o = orc.Oracle(nx=n, ny=n, nz=n, npart=npart, radius_um=SETS_UM, **PHYS)
    o.part_init()
    rng = np.random.default_rng(7)
    x = np.arange(n) * 2 * np.pi / n
    f = []
    for c in range(3):
        a = np.zeros((n, n, n + 2))
        a[:, :, :n] = (np.sin(x)[None, None, :] * np.cos(2 * x)[None, :, None] +
                       np.cos(x + c)[:, None, None])
        f.append(np.ascontiguousarray(a))
    o.update_step(*f)
    t = time.perf_counter()
    done = 0
    while done < steps or (time.perf_counter() - t) < min_seconds:
        o.update_step(*f)
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


def cpu_baseline():
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as orc
    npart = 200_000
    v, th, dt = _oracle_sample(npart, N_GRID, 3, min_seconds=10.0)
    orc.set_num_threads(1)
    n1 = 20_000
    v1, _, dt1 = _oracle_sample(n1, N_GRID, 3, min_seconds=4.0)
    orc.set_num_threads(th)
    flow_s = _cpu_flow_step()
    return {"value": v, "unit": "particle-updates/s", "cores": th, "kind": "port",
            "sample": f"{npart} droplets on the 256^3 FP64 field, >= 10 s of update steps "
                      f"(interpolation + history + advance + position), OpenMP over droplets; {dt:.3f} s/step",
            "cpu_model": _cpu_model(), "one_core_value": v1,
            "one_core_sample": f"{n1} droplets, 1 thread, {dt1:.3f} s/step",
            "flow_step_s_256": flow_s,
            "flow_sample": f"one 256^3 FP64 flow step of the numpy restatement with scipy.fft on {os.cpu_count()} "
                           f"workers"}


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
        ms, kms, launches = _time_update(g, stream, args.steps, args.warmup, torch)
        out.update(ms_per_step=ms, kernel_ms=kms, launches=launches)
        g.close()
    elif args.only == "adjoint":
        out.update(adjoint_bench(0, torch))
    elif args.only == "full":
        field = spectral_field(N_GRID, seed=1234, device="cuda:0")
        out.update(full_step_bench(0, torch, field))
    elif args.only == "config4":
        out.update(config4_bench(0, torch))
    print(json.dumps(out), flush=True)


def run_reference(args):
    ws, rank, local = _dist()
    if rank != 0:
        return
    npart = args.ref_sample
    for _ in range(args.warmup):
        pass
    v, th, dt = _oracle_sample(npart, N_GRID, args.steps)
    line = {
        "metric": "particle-updates/s (256^3, 1M droplets, mixed precision)", "impl": "reference",
        "value": v, "unit": "particle-updates/s", "n_gpus": ws, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": dt * 1e3 * N_PART / npart, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic", "config": CONFIG,
        "cpu_baseline": {"value": v, "unit": "particle-updates/s", "cores": th, "kind": "port",
                         "sample": f"{npart} droplets per step on the 256^3 field (FP64 CPU restatement "
                                   f"of partlib.f90; the Fortran/MPI reference cannot be built here)"},
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
    ap.add_argument("--ref-sample", type=int, default=200_000,
                    help="droplets per step of the reference arm's CPU sample")
    ap.add_argument("--only", choices=["update", "update-fp64", "adjoint", "full", "config4"],
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
