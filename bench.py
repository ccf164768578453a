#!/usr/bin/env python
"""Benchmark of the B200 LIMA_MD step path.

Workload: the 32,024-particle solvated-chain box (16 chains x 64 particles in
31,000 single-site solvents, 10 nm periodic box, 1.2 nm cutoff, Berendsen
300 K, dt 2 fs), seeded synthetic input.  One "step" is one MD step (forces,
integration, thermostat; the pair list is rebuilt, inside the step's CUDA
graph, whenever a particle has moved more than skin/2).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl reference]

Prints one JSON line.  value = simulated ns/day of the whole job (N
independent replicas under torchrun, one per GPU; device time, max over
ranks), L2 flushed before every timed step.  e2e = the same metric through the
public API from host arrays (box upload, K steps with per-step FP64 energy
readback, final positions).  --impl reference runs the reference's own step
code (oracle/_ref: Engine.cu built for the host) on the host cores.
"""
from __future__ import annotations

import argparse
import json
import math
import os
import statistics
import sys
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

WORKLOAD = "solvated_chains_32k"
SKIN = 0.1                # Verlet-list skin, nm
NS_PER_DAY_S = 86400.0   # seconds per day
FP32_NOMINAL_TFLOPS = 148 * 128 * 2 * 1.965e9 / 1e12   # clock-derived FP32 FMA peak (no measured figure)
FLOP_PER_PAIR = 32       # per unique pair within the cutoff (minimum image, r^2, rcp, LJ, force, both sides)


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=4000)
    ap.add_argument("--warmup", type=int, default=40)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default=WORKLOAD)
    ap.add_argument("--seed", type=int, default=2024)
    ap.add_argument("--cpu-sample-steps", type=int, default=2)
    ap.add_argument("--mode", default="full",
                    choices=["full", "kernels", "precision", "grad", "large", "large-fp64", "6lzm"],
                    help="kernels: only warm-up + K plain-FP32 steps (the command profiled with ncu); "
                         "precision: the NVE drift / force-error study of plain FP32 against mixed precision; "
                         "grad: the parameter-gradient study on the 8,192 LJ box; "
                         "large: the 258k solvated-chain box, mixed forward and adjoint gradients; "
                         "large-fp64: central differences of the FP64 oracle loss at the start state and "
                         "gradient that --mode large --grad-state saved (host only, no GPU); "
                         "6lzm: the reference's own demo box and settings, next to its published ms/step")
    ap.add_argument("--large-steps", type=int, default=10000, help="--mode large: mixed-precision forward steps")
    ap.add_argument("--nve-steps", type=int, default=50000, help="--mode precision: NVE steps per run")
    ap.add_argument("--eq-steps", type=int, default=5000, help="--mode precision: Berendsen equilibration steps")
    ap.add_argument("--replicas", type=int, default=1,
                    help="--mode precision: independent NVE starts (each a further --replica-gap Berendsen steps on)")
    ap.add_argument("--replica-gap", type=int, default=2500, help="--mode precision: steps between replica starts")
    ap.add_argument("--dts", default="2,1", help="--mode precision: time steps in fs, comma-separated")
    ap.add_argument("--grad-state", default="",
                    help="--mode large: save the gradient's start state, target and a 20-step adjoint gradient "
                         "here (.npz); --mode large-fp64: read it")
    ap.add_argument("--fd-workers", type=int, default=0, help="--mode large-fp64: host processes (0 = all cores)")
    ap.add_argument("--fp64-fd", action="store_true",
                    help="--mode grad: also central differences of the FP64 oracle loss (minutes of host time)")
    ap.add_argument("--semantics", default="physics", choices=["physics", "reference", "adjoint"],
                    help="--mode kernels: physics or reference steps, or one loss + adjoint pass over --steps steps")
    ap.add_argument("--log-every", type=int, default=0, help="--mode kernels, physics: frame log every N steps")
    ap.add_argument("--render", action="store_true", help="--mode kernels: render the final state once")
    ap.add_argument("--nlist-period", type=int, default=0,
                    help="--mode kernels, physics: 0 = list rebuilt on demand (conditional graph node), "
                         "P > 0 = every P steps")
    return ap.parse_args()


def run_kernels_only(args):
    """The profiled command: W + K steps of one engine, nothing else."""
    import torch
    from quantom_b200 import engine as E
    from quantom_b200 import systems as S
    if args.workload == "6lzm":   # the reference's demo box, as its input path builds it
        system = S.load_6lzm()
        spec = system.spec
    else:
        spec = S.CONFIGS[args.workload]
        system = S.make_system(args.workload, seed=args.seed)
    if args.semantics == "adjoint":
        # one loss + adjoint gradient pass: args.steps unrolled NVE steps, checkpoints every 10
        p = physics_params(E, spec, E.PRECISION_FP32, None, 0)
        p.thermostat = E.THERMOSTAT_NONE
        p.skin = 0.2
        with E.Engine(system, p) as eng:
            L, g = eng.grad(args.steps, 10, 50, 1.2 * 50 / 51, 1.0, 100.0, np.zeros(50))
            eng.synchronize()
            print(json.dumps({"mode": "kernels", "semantics": "adjoint", "steps": args.steps, "loss": L,
                              "grad": g.tolist()}), flush=True)
        return
    if args.semantics == "physics":
        p = physics_params(E, spec, E.PRECISION_FP32, None, 0)
        # a fixed period builds the step as a plain graph (profilers list its kernel nodes)
        p.nlist_period = args.nlist_period
    else:
        p = E.default_params(box_len=spec.box_len, cutoff=spec.cutoff, dt=spec.dt)
    with E.Engine(system, p) as eng:
        eng.step(max(3, args.warmup))
        eng.synchronize()
        if args.log_every > 0:   # frame log on (physics): k_log_frame / k_log_train at every logged step
            eng.log_start(args.log_every, ring_frames=16)
        eng.step(args.steps)
        eng.synchronize()
        if args.render:          # headless rasterizer: balls of the final state and a 1080 x 1080 image
            eng.render_image(1080, 1080)
        print(json.dumps({"mode": "kernels", "semantics": args.semantics, "steps": args.steps,
                          "ms_per_step_unflushed": eng.last_step_ms() / max(1, args.steps)}), flush=True)


def dist_setup(args, backend="nccl", timeout_s=120):
    """One process per GPU (torchrun's RANK / LOCAL_RANK / WORLD_SIZE): the
    replicas share only a barrier and the max of their step times.  backend
    "gloo" runs the same plumbing on host processes."""
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    pg = None
    if ws > 1:
        import datetime
        import torch.distributed as dist
        os.environ.setdefault("MASTER_ADDR", "127.0.0.1")
        if backend == "nccl":
            import torch
            torch.cuda.set_device(local)
        dist.init_process_group(backend, timeout=datetime.timedelta(seconds=timeout_s))
        pg = dist
    return ws, rank, local, pg


def max_over_ranks(x, pg, device):
    if pg is None:
        return x
    import torch
    t = torch.tensor([x], dtype=torch.float64, device=device)
    pg.all_reduce(t, op=pg.ReduceOp.MAX)
    return float(t.item())


def barrier(pg):
    if pg is not None:
        pg.barrier()


class ClockSampler:
    """SM clock and clock-event reasons sampled every 10 ms through NVML
    (read-only queries) by a background thread, plus one sample at the entry
    and one at the exit of the timed window, so a window shorter than the
    period still has samples; `window()` brackets the timed region and
    `summary()` keeps the samples taken inside it."""
    REASONS = (("hw_slowdown", 0x8), ("hw_thermal_slowdown", 0x40), ("sw_thermal_slowdown", 0x20),
               ("sw_power_cap", 0x4), ("hw_power_brake_slowdown", 0x80))

    def __init__(self, device, period_s=0.01):
        self.device = device
        self._sample = None
        self.period = period_s
        self.samples = []          # (t, sm_mhz, reasons bitmask, power W)
        self.win = [None, None]
        self.sm_max = None
        self._stop = None
        self._thr = None

    def _handle(self, nv):
        import torch
        try:
            pr = torch.cuda.get_device_properties(self.device)
            bus = f"{pr.pci_domain_id:08x}:{pr.pci_bus_id:02x}:{pr.pci_device_id:02x}.0"
            return nv.nvmlDeviceGetHandleByPciBusId(bus)
        except Exception:
            return nv.nvmlDeviceGetHandleByIndex(self.device)

    def __enter__(self):
        import threading
        try:
            import pynvml as nv
            nv.nvmlInit()
            h = self._handle(nv)
            self.sm_max = float(nv.nvmlDeviceGetMaxClockInfo(h, nv.NVML_CLOCK_SM))
        except Exception:
            return self
        self._stop = threading.Event()

        def sample():
            try:
                t = time.perf_counter()
                sm = float(nv.nvmlDeviceGetClockInfo(h, nv.NVML_CLOCK_SM))
                rs = int(nv.nvmlDeviceGetCurrentClocksEventReasons(h))
                pw = nv.nvmlDeviceGetPowerUsage(h) / 1000.0
                self.samples.append((t, sm, rs, pw))
            except Exception:
                pass
        self._sample = sample

        def loop():
            while not self._stop.is_set():
                sample()
                self._stop.wait(self.period)

        self._thr = threading.Thread(target=loop, daemon=True)
        self._thr.start()
        return self

    def window(self):
        s = self

        class _W:
            def __enter__(self_):
                s.win[0] = time.perf_counter()
                if s._sample:
                    s._sample()   # one sample at the window's entry, whatever the period

            def __exit__(self_, *a):
                if s._sample:
                    s._sample()   # and one at its exit, before the window closes
                s.win[1] = time.perf_counter()
        return _W()

    def __exit__(self, *a):
        if self._thr is not None:
            self._stop.set()
            self._thr.join(timeout=5)
            try:
                import pynvml as nv
                nv.nvmlShutdown()
            except Exception:
                pass

    def summary(self):
        t0, t1 = self.win
        inside = [x for x in self.samples if t0 is not None and t0 <= x[0] <= (t1 or t0)]
        reasons = sorted({nm for x in inside for nm, bit in self.REASONS if x[2] & bit})
        return {"sm_mhz": statistics.median([x[1] for x in inside]) if inside else None,
                "sm_max_mhz": self.sm_max, "reasons": reasons, "samples": len(inside),
                "power_w_median": statistics.median([x[3] for x in inside]) if inside else None,
                "source": "NVML, every 10 ms during the timed steps and at the window's entry and exit"}


def measured_peaks():
    try:
        return json.loads((ROOT / "MEASURED_PEAKS.json").read_text())
    except Exception:
        return {}


def ncu_traffic(kernel, workload):
    """dram bytes per launch from the committed ncu summary, if present."""
    p = ROOT / "profiles" / f"ncu_{kernel}_{workload}.md"
    if not p.exists():
        return None
    for line in p.read_text().splitlines():
        if line.strip().startswith("dram_bytes_per_launch:"):
            try:
                return float(line.split(":", 1)[1].strip().split()[0])
            except ValueError:
                return None
    return None


def physics_params(E, spec, precision, stream_handle=None, device=0, dt=None):
    p = E.default_params(box_len=spec.box_len, cutoff=spec.cutoff, dt=spec.dt if dt is None else dt,
                         semantics=E.SEMANTICS_PHYSICS,
                         precision=precision, skin=SKIN, switch_on=1.0, nlist_period=0, t_target=spec.temperature,
                         tau_t=spec.tau_t, device=device)
    p.thermostat = E.THERMOSTAT_BERENDSEN if spec.thermostat == "berendsen" else E.THERMOSTAT_NONE
    if stream_handle is not None:
        p.stream = stream_handle
    return p


def timed_steps(eng, stream, n, flush):
    """Device time of n steps, L2 flushed (untimed) before each."""
    import torch
    evs = []
    for _ in range(n):
        with torch.cuda.stream(stream):
            flush.zero_()
        a = torch.cuda.Event(enable_timing=True)
        b = torch.cuda.Event(enable_timing=True)
        a.record(stream)
        eng.step(1)
        b.record(stream)
        evs.append((a, b))
    stream.synchronize()
    eng.synchronize()
    return sum(a.elapsed_time(b) for a, b in evs)   # ms


def ns_per_day(dt_ns, ms_per_step):
    return dt_ns * NS_PER_DAY_S / (ms_per_step * 1e-3)


# ------------------------------------------------------- precision study --
K_B = 8.314462618        # J/(mol K)


def with_state(system, st, prev, sol):
    """The same topology with positions/previous positions from a readback."""
    import copy
    s = copy.copy(system)
    s.compounds = system.compounds.copy()
    s.states = system.states.copy()
    s.solvents = sol.copy()
    for c in range(system.n_compounds):
        s.states[c]["positions"] = st[c]["positions"]
        s.compounds[c]["prev_positions"] = prev[c]
    return s


def rescale_dt(system, factor):
    """Previous positions for a time step `factor` times the current one
    (same velocities: x_prev' = x - factor * (x - x_prev))."""
    import copy
    s = copy.copy(system)
    s.compounds = system.compounds.copy()
    s.solvents = system.solvents.copy()
    for c in range(system.n_compounds):
        x = system.states[c]["positions"].astype(np.float64)
        xp = system.compounds[c]["prev_positions"].astype(np.float64)
        s.compounds[c]["prev_positions"] = (x - factor * (x - xp)).astype(np.float32)
    x = system.solvents["pos"].astype(np.float64)
    xp = system.solvents["pos_tsub1"].astype(np.float64)
    s.solvents["pos_tsub1"] = (x - factor * (x - xp)).astype(np.float32)
    return s


def flat_forces(system, fc, fs):
    parts = [fc[c, : system.compounds[c]["n_particles"]] for c in range(system.n_compounds)]
    return np.concatenate(parts + [fs]) if parts else fs


def drift_fit(t, e):
    """Least-squares slope of e(t) and its standard error, the latter widened
    for correlated residuals: SE = sigma_r * sqrt(tau / sum (t - mean t)^2),
    tau = 1 + 2 * sum of the residual autocorrelation up to its first
    negative lag (integrated autocorrelation time, in samples)."""
    coef = np.polyfit(t, e, 1)
    r = e - np.polyval(coef, t)
    n = len(r)
    var = float(r.var())
    tau = 1.0
    if var > 0:
        for k in range(1, n // 2):
            rho = float(np.dot(r[:-k], r[k:]) / ((n - k) * var))
            if rho <= 0:
                break
            tau += 2 * rho
    se = math.sqrt(var * tau / float(((t - t.mean()) ** 2).sum()))
    return float(coef[0]), se, tau


def run_precision(args):
    """Config-2 study on the 32k box: Berendsen equilibration, then NVE runs
    of plain FP32 and mixed precision at dt 2 fs and 1 fs from each of
    --replicas starts (the equilibration continued --replica-gap steps
    between starts).  Drift = slope of a linear fit of the total energy, per
    particle, in kT per ns; per precision and dt the replicas' mean, with the
    larger of two standard errors of that mean (the fits' errors combined,
    and the replicas' scatter / sqrt(R) when R > 1).  Force error = relative
    RMS against the FP64 oracle at the same positions."""
    from oracle import pyoracle as po
    from quantom_b200 import engine as E
    from quantom_b200 import systems as S
    spec = S.CONFIGS[args.workload]
    system = S.make_system(args.workload, seed=args.seed)
    n = system.n_particles
    kT = K_B * spec.temperature
    R = max(1, args.replicas)
    starts = []
    with E.Engine(system, physics_params(E, spec, E.PRECISION_FP32)) as eq:
        eq.step(args.eq_steps)
        for r in range(R):
            if r:
                eq.step(args.replica_gap)
            st, prev = eq.compound_states()
            starts.append(with_state(system, st, prev, eq.solvents()))
    start = starts[0]

    def force_errors(sys_x):
        F64, _ = po.PhysSystem(sys_x, rc=spec.cutoff, r_on=1.0).forces()
        out = {}
        for name, prec in (("fp32", E.PRECISION_FP32), ("mixed", E.PRECISION_MIXED)):
            p = physics_params(E, spec, prec)
            p.thermostat = E.THERMOSTAT_NONE
            with E.Engine(sys_x, p) as eng:
                eng.compute_energies()
                F = flat_forces(sys_x, *eng.forces()).astype(np.float64)
            out[name] = float(np.sqrt(((F - F64) ** 2).sum() / (F64 ** 2).sum()))
        return out

    result = {"mode": "precision", "workload": args.workload, "particles": n, "eq_steps": args.eq_steps,
              "nve_steps": args.nve_steps, "replicas": R, "replica_gap_steps": args.replica_gap,
              "force_relrms_vs_fp64": {"start": force_errors(start)}, "runs": []}
    block = 100
    end = None
    dts = [float(x) for x in args.dts.split(",")]
    result["dts_fs"] = dts
    for r, start_r in enumerate(starts):
        for dt_fs in dts:
            sys_dt = rescale_dt(start_r, dt_fs * 1e-6 / spec.dt)
            for name, prec in (("fp32", E.PRECISION_FP32), ("mixed", E.PRECISION_MIXED)):
                p = physics_params(E, spec, prec, dt=dt_fs * 1e-6)
                p.thermostat = E.THERMOSTAT_NONE
                t_ns, etot, temp = [], [], []
                with E.Engine(sys_dt, p) as eng:
                    for b in range(args.nve_steps // block + 1):
                        e = eng.compute_energies()
                        t_ns.append(b * block * dt_fs * 1e-6)
                        etot.append(e[E.E_TOTAL])
                        temp.append(e[E.E_TEMPERATURE])
                        if b < args.nve_steps // block:
                            eng.step(block)
                    if r == 0 and dt_fs == dts[0] and name == "fp32":
                        st2, prev2 = eng.compound_states()
                        end = with_state(system, st2, prev2, eng.solvents())
                t = np.asarray(t_ns)
                et = np.asarray(etot)
                slope, se, tau = drift_fit(t, et)
                resid = et - np.polyval(np.polyfit(t, et, 1), t)
                result["runs"].append({
                    "replica": r, "precision": name, "dt_fs": dt_fs, "simulated_ps": float(t[-1] * 1e3),
                    "drift_kT_per_particle_per_ns": slope / (n * kT),
                    "drift_stderr_kT_per_particle_per_ns": se / (n * kT),
                    "residual_autocorr_samples": tau,
                    "drift_J_per_mol_per_ns": slope,
                    "etot_fluct_rms_kT_per_particle": float(resid.std() / (n * kT)),
                    "temperature_mean_K": float(np.mean(temp)), "temperature_first_last_K": [temp[0], temp[-1]],
                })
                print(json.dumps(result["runs"][-1]), flush=True)
    result["force_relrms_vs_fp64"][f"after_nve_fp32_{dts[0]:g}fs"] = force_errors(end)
    # Per precision and dt over the replicas: the signed mean drift, and the
    # mean drift magnitude |slope|.  The FP32 energy wanders like a random
    # walk whose sign differs between replicas, so the ratio is taken on the
    # magnitudes; its standard errors are the larger of the fits' combined
    # errors and the replicas' scatter / sqrt(R).
    combined = {}
    for dt_fs in dts:
        for name in ("fp32", "mixed"):
            runs = [x for x in result["runs"] if x["dt_fs"] == dt_fs and x["precision"] == name]
            d = np.array([x["drift_kT_per_particle_per_ns"] for x in runs])
            a = np.abs(d)
            se_fit = math.sqrt(sum(x["drift_stderr_kT_per_particle_per_ns"] ** 2 for x in runs)) / len(runs)
            se_scatter = float(d.std(ddof=1) / math.sqrt(len(d))) if len(d) > 1 else 0.0
            se_abs_scatter = float(a.std(ddof=1) / math.sqrt(len(a))) if len(a) > 1 else 0.0
            combined[(dt_fs, name)] = (float(a.mean()), max(se_fit, se_abs_scatter), float(d.mean()),
                                       max(se_fit, se_scatter))
            result.setdefault("combined", []).append({
                "precision": name, "dt_fs": dt_fs, "replicas": len(runs),
                "simulated_ps_total": float(sum(x["simulated_ps"] for x in runs)),
                "drift_kT_per_particle_per_ns": float(d.mean()),
                "drift_stderr": max(se_fit, se_scatter),
                "drift_magnitude_kT_per_particle_per_ns": float(a.mean()),
                "drift_magnitude_stderr": max(se_fit, se_abs_scatter),
                "stderr_fits": se_fit, "stderr_replica_scatter": se_scatter,
                "stderr_magnitude_replica_scatter": se_abs_scatter})
        (d32, s32, _, _), (dmx, smx, mmx, smm) = combined[(dt_fs, "fp32")], combined[(dt_fs, "mixed")]
        result[f"drift_ratio_fp32_over_mixed_{int(dt_fs)}fs"] = d32 / max(dmx, 1e-30)
        # lower bound: FP32 magnitude less 2 standard errors over mixed magnitude plus 2 standard errors
        result[f"drift_ratio_lower_bound_2se_{int(dt_fs)}fs"] = max(d32 - 2 * s32, 0.0) / (dmx + 2 * smx)
        # the same against the mixed runs' systematic drift (their signed mean; its random part averages out)
        result[f"drift_ratio_lower_bound_2se_vs_mixed_signed_mean_{int(dt_fs)}fs"] = (
            max(d32 - 2 * s32, 0.0) / (abs(mmx) + 2 * smm))
    print(json.dumps(result), flush=True)


# ----------------------------------------------------- parameter gradients --
GRAD_WORKLOAD = "lj_solvent_8192"


def grad_study(E, S, device=0, fd=True, fp64_fd=False):
    """Config-3 gradient: 8,192 LJ particles in a 6.3 nm box, loss = <U>/N +
    RDF-bin loss (50 bins over 0..r_max, support ending at the 1.2 nm cutoff)
    over a 200-step NVE unroll with checkpoints every 20 steps.  Returns cost
    and accuracy figures."""
    import torch
    spec = S.CONFIGS[GRAD_WORKLOAD]
    system = S.make_system(GRAD_WORKLOAD, seed=2024)
    nb, rmax, T, C = 50, 1.2 * 50 / 51, 200, 20
    w_e, w_r = 1.0, 100.0

    def params(thermostat):
        p = E.default_params(box_len=spec.box_len, cutoff=spec.cutoff, dt=spec.dt, semantics=E.SEMANTICS_PHYSICS,
                             precision=E.PRECISION_FP32, skin=0.2, switch_on=1.0, nlist_period=0,
                             t_target=300.0, tau_t=1e-4, device=device)
        p.thermostat = thermostat
        return p

    # equilibrate, then a target occupancy from the same box with sigma + 2 %
    with E.Engine(system, params(E.THERMOSTAT_BERENDSEN)) as eq:
        eq.step(3000)
        st, prev = eq.compound_states()
        sol = eq.solvents()
        start = system.with_state(st, prev, sol)
        th = eq.get_params()
        th2 = th.copy()
        th2[0] *= 1.02
        eq.set_params(th2)
        eq.step(1000)
        target = np.zeros(nb)
        for _ in range(10):
            eq.step(50)
            target += eq.rdf(nb, rmax) / 10
    out = {"workload": f"{GRAD_WORKLOAD}: {system.n_particles} particles, {spec.box_len} nm box, rc 1.2 nm "
                       f"(C2 switch from 1.0), skin 0.2 nm, NVE dt 2 fs, FP32",
           "n_steps": T, "checkpoint_every": C, "n_bins": nb, "r_max_nm": rmax, "w_energy": w_e, "w_rdf": w_r,
           "target": "RDF-bin occupancy of the same box equilibrated with sigma + 2 %"}
    with E.Engine(start, params(E.THERMOSTAT_NONE)) as eng:
        theta = eng.get_params()

        def wall(fn, reps=3):
            fn()
            torch.cuda.synchronize(device)
            ts = []
            for _ in range(reps):
                t0 = time.perf_counter()
                r = fn()
                torch.cuda.synchronize(device)
                ts.append(time.perf_counter() - t0)
            return r, 1e3 * min(ts)
        L, t_loss = wall(lambda: eng.loss(T, C, nb, rmax, w_e, w_r, target))
        (L2, g), t_grad = wall(lambda: eng.grad(T, C, nb, rmax, w_e, w_r, target))
        (_, g1), t_grad1 = wall(lambda: eng.grad(T, T, nb, rmax, w_e, w_r, target))   # one segment: every state kept
        out.update({"loss": L, "theta": theta.tolist(), "grad": g.tolist(), "ms_forward_loss": t_loss,
                    "ms_grad": t_grad, "grad_over_forward": t_grad / t_loss, "ms_grad_all_states_kept": t_grad1,
                    "grad_all_states_kept_over_forward": t_grad1 / t_loss,
                    "loss_same_in_both_calls": abs(L2 - L) <= 1e-9 * abs(L)})
        if fd:
            # central differences of the FP32 GPU loss at the specified step (1e-4 relative) and
            # at 1e-3, where the trajectories' FP32 rounding noise weighs 10x less
            for hrel, key in ((1e-4, ""), (1e-3, "_h1e-3")):
                fdv, rel = [], []
                for k in (0, 1):   # sigma and epsilon of the one LJ type
                    h = hrel * abs(theta[k])
                    tp = theta.copy()
                    tp[k] += h
                    eng.set_params(tp)
                    lp = eng.loss(T, C, nb, rmax, w_e, w_r, target)
                    tp[k] -= 2 * h
                    eng.set_params(tp)
                    lm = eng.loss(T, C, nb, rmax, w_e, w_r, target)
                    eng.set_params(theta)
                    fdv.append((lp - lm) / (2 * h))
                    rel.append(abs(g[k] - fdv[-1]) / abs(fdv[-1]))
                out.update({"fd_fp32_gpu" + key: fdv, "rel_err_vs_fd_fp32_gpu" + key: rel})
    if fp64_fd:
        # central differences of the FP64 oracle loss at the specified step (1e-4
        # relative), the four losses in parallel host processes
        import multiprocessing as mp
        from concurrent.futures import ProcessPoolExecutor
        from oracle import pyoracle as po
        t0 = time.perf_counter()
        ps = po.PhysSystem(start, rc=spec.cutoff, r_on=1.0)
        th64 = ps.params()
        jobs, hs = [], []
        for k in (0, 1):
            h = 1e-4 * abs(th64[k])
            hs.append(h)
            for sign in (1.0, -1.0):
                e = np.zeros(len(th64))
                e[k] = sign * h
                jobs.append((ps, th64 + e, spec.dt, T, nb, rmax, w_e, w_r, target))
        with ProcessPoolExecutor(min(4, os.cpu_count() or 1), mp_context=mp.get_context("spawn")) as ex:
            losses = list(ex.map(_fp64_loss, jobs))
        fdv = [(losses[2 * k] - losses[2 * k + 1]) / (2 * hs[k]) for k in (0, 1)]
        rel = [abs(g[k] - fdv[k]) / abs(fdv[k]) for k in (0, 1)]
        out.update({"fd_fp64_oracle": fdv, "rel_err_vs_fd_fp64": rel, "fd_fp64_host_s": time.perf_counter() - t0})
    return out


def _fp64_loss(job):
    """One FP64 oracle loss (a spawn-pool task of the gradient check)."""
    ps, theta, dt, T, nb, rmax, w_e, w_r, target = job
    return ps.with_params(theta).loss(dt, T, nb, rmax, w_e, w_r, target)[0]


def run_grad(args):
    from quantom_b200 import engine as E
    from quantom_b200 import systems as S
    print(json.dumps({"mode": "grad", **grad_study(E, S, fp64_fd=args.fp64_fd)}), flush=True)


# ------------------------------------------------- large solvated chains --
LARGE_WORKLOAD = "solvated_chains_258k"


def run_large(args):
    """The 258k box: 64 chains x 128 particles (two compounds and one
    bridge each) in 250,000 solvents, 20 nm box, rc 1.2 nm.  Mixed-precision
    forward (Berendsen 300 K, tau 0.1 ps) for --large-steps steps: device time
    of the whole run (one event pair; the pair list alone is larger than the
    L2), ns/day, list rebuilds; forces of the first state against the FP64
    oracle.  Then the adjoint gradient of <U>/N + 100 x RDF-bin loss over a
    100-step NVE unroll with checkpoints every 10 with respect to sigma and
    epsilon of every type (solvent and the 4 chain types) and the bond,
    angle and dihedral scales; its cost against the forward loss; central
    differences of the FP32 GPU loss (step 1e-3 relative) for every
    component."""
    import torch
    from oracle import pyoracle as po
    from quantom_b200 import engine as E
    from quantom_b200 import systems as S
    spec = S.CONFIGS[LARGE_WORKLOAD]
    t0 = time.perf_counter()
    system = S.make_system(LARGE_WORKLOAD, seed=args.seed)
    t_gen = time.perf_counter() - t0
    n = system.n_particles
    dev = torch.device("cuda", 0)
    stream = torch.cuda.Stream(device=dev)
    out = {"mode": "large", "workload": f"{LARGE_WORKLOAD}: 64 chains x 128 (2 compounds + 1 bridge each) + "
                                        f"250,000 solvents, {spec.box_len} nm box, rc 1.2 nm (C2 switch from 1.0), "
                                        f"skin {SKIN} nm, dynamic lists, Berendsen 300 K tau 0.1 ps, dt 2 fs",
           "particles": n, "compounds": system.n_compounds, "bridges": int(len(system.bridges)),
           "generate_s": t_gen}

    def params(prec, thermostat, skin=SKIN):
        p = physics_params(E, spec, prec, stream.cuda_stream, 0)
        p.thermostat = thermostat
        p.skin = skin
        return p

    # forces of the generated state against the FP64 oracle
    F64, en64 = po.PhysSystem(system, rc=spec.cutoff, r_on=1.0).forces()
    for name, prec in (("fp32", E.PRECISION_FP32), ("mixed", E.PRECISION_MIXED)):
        with E.Engine(system, params(prec, E.THERMOSTAT_NONE)) as eng:
            tot = eng.compute_energies()
            F = flat_forces(system, *eng.forces()).astype(np.float64)
        out[f"force_relrms_vs_fp64_{name}"] = float(np.sqrt(((F - F64) ** 2).sum() / (F64 ** 2).sum()))
        out[f"lj_energy_rel_err_{name}"] = abs(tot[E.E_LJ] - en64[0]) / abs(en64[0])

    # mixed-precision forward from the generated state; then, from where it ended,
    # mixed and plain FP32 side by side over the same number of steps
    start = system
    short = max(1000, args.large_steps // 5)
    for name, prec, steps in (("mixed", E.PRECISION_MIXED, args.large_steps),
                              ("mixed_equilibrated", E.PRECISION_MIXED, short), ("fp32", E.PRECISION_FP32, short)):
        with E.Engine(start, params(prec, E.THERMOSTAT_BERENDSEN)) as eng:
            eng.step(max(3, args.warmup))
            eng.synchronize()
            r0 = eng.rebuild_count()
            a = torch.cuda.Event(enable_timing=True)
            b = torch.cuda.Event(enable_timing=True)
            a.record(stream)
            eng.step(steps)
            b.record(stream)
            stream.synchronize()
            eng.synchronize()
            ms = a.elapsed_time(b) / steps
            e = eng.compute_energies()
            out[name] = {"steps": steps, "ms_per_step": ms, "ns_per_day": ns_per_day(spec.dt, ms),
                         "steps_per_list_rebuild": steps / max(1, eng.rebuild_count() - r0),
                         "temperature_end_K": e[E.E_TEMPERATURE], "kernels_ms": eng.profile_steps(100)}
            if name == "mixed":
                st, prev = eng.compound_states()
                start = system.with_state(st, prev, eng.solvents())
        print(json.dumps({name: out[name]}), flush=True)
    out["mixed_over_fp32"] = out["mixed_equilibrated"]["ms_per_step"] / out["fp32"]["ms_per_step"]

    # adjoint gradient over a 100-step NVE unroll
    T, C, nb, rmax, w_e, w_r = 100, 10, 50, 1.2 * 50 / 51, 1.0, 100.0
    with E.Engine(start, params(E.PRECISION_FP32, E.THERMOSTAT_BERENDSEN, skin=0.2)) as eq:
        th = eq.get_params()
        th2 = th.copy()
        th2[0] *= 1.02
        eq.set_params(th2)
        eq.step(500)
        target = np.zeros(nb)
        for _ in range(5):
            eq.step(20)
            target += eq.rdf(nb, rmax) / 5
    with E.Engine(start, params(E.PRECISION_FP32, E.THERMOSTAT_NONE, skin=0.2)) as eng:
        theta = eng.get_params()

        def wall(fn, reps=3):
            fn()
            torch.cuda.synchronize(dev)
            ts = []
            for _ in range(reps):
                t1 = time.perf_counter()
                r = fn()
                torch.cuda.synchronize(dev)
                ts.append(time.perf_counter() - t1)
            return r, 1e3 * min(ts)
        L, t_loss = wall(lambda: eng.loss(T, C, nb, rmax, w_e, w_r, target))
        (_, g), t_grad = wall(lambda: eng.grad(T, C, nb, rmax, w_e, w_r, target))
        fds, rels = {}, {}
        for step in (1e-3, 1e-2):
            fd, rel = [], []
            for k in range(len(theta)):
                h = step * abs(theta[k]) if theta[k] != 0.0 else step   # a zero phase: step in rad
                tp = theta.copy()
                tp[k] += h
                eng.set_params(tp)
                lp = eng.loss(T, C, nb, rmax, w_e, w_r, target)
                tp[k] -= 2 * h
                eng.set_params(tp)
                lm = eng.loss(T, C, nb, rmax, w_e, w_r, target)
                eng.set_params(theta)
                fd.append((lp - lm) / (2 * h))
                rel.append(abs(g[k] - fd[-1]) / max(abs(fd[-1]), 1e-300))
            fds[step], rels[step] = fd, rel
        names = eng.param_names()
        out["grad"] = {"n_steps": T, "checkpoint_every": C, "n_bins": nb, "w_energy": w_e, "w_rdf": w_r,
                       "target": "RDF-bin occupancy of the same box run with solvent sigma + 2 %",
                       "loss": L, "ms_forward_loss": t_loss, "ms_grad": t_grad, "grad_over_forward": t_grad / t_loss,
                       "params": names, "theta": theta.tolist(), "grad": g.tolist(),
                       "fd_fp32_gpu_h1e-3": fds[1e-3], "rel_err_vs_fd_h1e-3": rels[1e-3],
                       "fd_fp32_gpu_h1e-2": fds[1e-2], "rel_err_vs_fd_h1e-2": rels[1e-2]}
        if args.grad_state:
            # the FP64 pin: a 20-step unroll from the same state, gradient kept with the state
            # for --mode large-fp64 (the oracle's loss costs ~20 s of host time per step here)
            T64 = 20
            L64, g64 = eng.grad(T64, C, nb, rmax, w_e, w_r, target)
            np.savez(args.grad_state, forcefield=start.forcefield, compounds=start.compounds, states=start.states,
                     solvents=start.solvents, bridges=start.bridges, target=target, theta=theta, grad=g64,
                     loss=L64, names=np.array(names), n_steps=T64, checkpoint_every=C, n_bins=nb, r_max=rmax,
                     w_energy=w_e, w_rdf=w_r, dt=spec.dt, cutoff=spec.cutoff, seed=args.seed)
            out["grad"]["saved_for_fp64_check"] = {"path": args.grad_state, "n_steps": T64, "loss": L64}
    print(json.dumps(out), flush=True)


def _fd64_one(job):
    """One central difference of the FP64 oracle loss (a spawn-pool task)."""
    from oracle import pyoracle as po
    system, k, h, a = job
    ps = po.PhysSystem(system, rc=a["cutoff"], r_on=1.0)
    th = ps.params()
    e = np.zeros(len(th))
    e[k] = h
    lp, _ = ps.with_params(th + e).loss(a["dt"], a["n_steps"], a["n_bins"], a["r_max"], a["w_energy"], a["w_rdf"],
                                        a["target"])
    lm, _ = ps.with_params(th - e).loss(a["dt"], a["n_steps"], a["n_bins"], a["r_max"], a["w_energy"], a["w_rdf"],
                                        a["target"])
    return (lp - lm) / (2 * h)


def run_large_fp64(args):
    """The 258k box's adjoint gradient (saved by --mode large --grad-state)
    against central differences of the FP64 oracle loss (oracle/lima_oracle.c
    orc_phys_loss) over the same unroll, every entry of theta, step 1e-4
    relative (1e-4 rad for a zero phase); host processes only."""
    import multiprocessing as mp
    from concurrent.futures import ProcessPoolExecutor
    from oracle import pyoracle as po
    from quantom_b200 import systems as S
    z = np.load(args.grad_state)
    spec = S.CONFIGS[LARGE_WORKLOAD]
    system = S.System(spec, int(z["seed"]), z["forcefield"], z["compounds"], z["states"], z["solvents"],
                      z["bridges"])
    a = {k: (z[k] if k == "target" else float(z[k])) for k in
         ("target", "dt", "cutoff", "r_max", "w_energy", "w_rdf")}
    a.update({k: int(z[k]) for k in ("n_steps", "n_bins")})
    theta, g, names = z["theta"], z["grad"], [str(x) for x in z["names"]]
    th64 = po.PhysSystem(system, rc=a["cutoff"], r_on=1.0).params()
    steps = [1e-4 * abs(v) if v != 0.0 else 1e-4 for v in th64]
    workers = args.fd_workers or os.cpu_count() or 1
    t0 = time.perf_counter()
    with ProcessPoolExecutor(workers, mp_context=mp.get_context("spawn")) as ex:
        fd = np.array(list(ex.map(_fd64_one, [(system, k, steps[k], a) for k in range(len(th64))])))
    rel = np.abs(g - fd) / np.maximum(np.abs(fd), 1e-300)
    print(json.dumps({"mode": "large-fp64", "workload": LARGE_WORKLOAD, "n_steps": a["n_steps"],
                      "theta_matches_oracle": bool(np.allclose(theta, th64, rtol=1e-6)), "params": names,
                      "grad_adjoint_fp32": g.tolist(), "fd_fp64_oracle": fd.tolist(), "rel_err": rel.tolist(),
                      "max_rel_err": float(rel.max()), "host_workers": workers,
                      "host_s": time.perf_counter() - t0}), flush=True)


# ------------------------------------------------------- the reference's demo --
PUBLISHED_6LZM_MS = 3.34   # README.md:19: LIMA_MD ms/step on this box, RTX 2080 Ti, all features on


def run_6lzm(args):
    """The reference's own benchmark system: T4 lysozyme (6LZM) heavy atoms in
    36 compounds + 35 bridges and 5,000 single-site waters in a 7 nm box, as the
    reference's input path builds it (the native builder reproduces it bit for
    bit), with the settings of its published run: CUTOFF 0.7 nm, dt 0.1 fs,
    lists every 200 steps, its thermostat every 40 steps.  Device time per step
    with the L2 flushed before every step, next to the published 3.34 ms/step
    (RTX 2080 Ti).  Also the physics semantics on the same box (cutoff 1.4 nm
    with a C2 switch from 1.0, skin 0.1 nm, dynamic lists, NVE)."""
    import torch
    from oracle import pyoracle as po
    from quantom_b200 import engine as E
    from quantom_b200 import systems as S
    system = S.load_6lzm()
    spec = system.spec
    dev = torch.device("cuda", 0)
    stream = torch.cuda.Stream(device=dev)
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device=dev)
    steps = max(200, args.steps)
    out = {"mode": "6lzm", "workload": "6lzm: T4 lysozyme heavy atoms (1,293 in 36 compounds, 35 bridges) + 5,000 "
                                       "waters, 7 nm box, dt 0.1 fs", "particles": system.n_particles,
           "steps": steps, "published_reference_ms_per_step": PUBLISHED_6LZM_MS,
           "published_hardware": "RTX 2080 Ti (README.md:19)"}
    p = E.default_params(box_len=spec.box_len, cutoff=spec.cutoff, dt=spec.dt, device=0)
    p.thermostat = E.THERMOSTAT_REFERENCE
    p.t_target = 310.0
    p.stream = stream.cuda_stream
    with E.Engine(system, p) as eng:
        timed_steps(eng, stream, max(3, args.warmup), flush)
        ms = timed_steps(eng, stream, steps, flush) / steps
        out["reference_semantics"] = {"ms_per_step": ms, "speedup_vs_published": PUBLISHED_6LZM_MS / ms,
                                      "kernels_ms": eng.profile_steps(50),
                                      "settings": "CUTOFF 0.7 nm (lists within 2 CUTOFF), lists every 200 steps, "
                                                  "reference thermostat every 40 steps, FP32"}
    print(json.dumps({"reference_semantics": out["reference_semantics"]}), flush=True)
    pp = E.default_params(box_len=spec.box_len, cutoff=spec.cutoff, dt=spec.dt, semantics=E.SEMANTICS_PHYSICS,
                          skin=SKIN, switch_on=1.0, nlist_period=0, device=0)
    pp.stream = stream.cuda_stream
    F64, _ = po.PhysSystem(system, rc=spec.cutoff, r_on=1.0).forces()
    with E.Engine(system, pp) as eng:
        eng.compute_energies()
        F = flat_forces(system, *eng.forces()).astype(np.float64)
        timed_steps(eng, stream, max(3, args.warmup), flush)
        ms = timed_steps(eng, stream, steps, flush) / steps
        out["physics_semantics"] = {"ms_per_step": ms, "speedup_vs_published": PUBLISHED_6LZM_MS / ms,
                                    "force_relrms_vs_fp64": float(np.sqrt(((F - F64) ** 2).sum() / (F64 ** 2).sum())),
                                    "kernels_ms": eng.profile_steps(50)}
    print(json.dumps(out), flush=True)


def c0_study(E, S, stream, flush, device):
    """The reference's CPU-runnable case (4,096 single-site waters, 5 nm box,
    rc 1.2 nm, dt 2 fs, NVE): the physics step on the GPU, and the reference's
    own step code and neighbour-list update on the host cores, timed apart."""
    spec = S.CONFIGS["lj_solvent_4096"]
    system = S.make_system("lj_solvent_4096", seed=2024)
    with E.Engine(system, physics_params(E, spec, E.PRECISION_FP32, stream.cuda_stream, device)) as eng:
        timed_steps(eng, stream, 20, flush)
        ms = timed_steps(eng, stream, spec.n_steps, flush) / spec.n_steps
        prof = eng.profile_steps(50)
    threads = os.cpu_count() or 1
    per_step, t_step, t_nl, kind, used = cpu_reference_rate(system, 20, threads)
    _, t_step1, t_nl1, _, used1 = cpu_reference_rate(system, 5, 1)
    return {"workload": f"lj_solvent_4096: {system.n_particles} waters, {spec.box_len} nm box, rc 1.2 nm (C2 switch "
                        f"from 1.0), skin 0.1 nm, NVE, dt 2 fs, {spec.n_steps} timed steps, L2 flushed before each",
            "gpu_ms_per_step": ms, "gpu_ns_per_day": ns_per_day(spec.dt, ms), "gpu_kernels_ms": prof,
            "cpu": {"kind": kind, "cores": used, "force_integrate_ms_per_step": t_step * 1e3,
                    "nlist_update_ms": t_nl * 1e3, "ns_per_day_list_every_200": ns_per_day(spec.dt, per_step * 1e3),
                    "sample": "20 steps of the reference's own step code (reference semantics) and one neighbour-list "
                              "update",
                    "one_thread": {"cores": used1, "force_integrate_ms_per_step": t_step1 * 1e3,
                                   "nlist_update_ms": t_nl1 * 1e3}}}


# --------------------------------------------------------------- CPU side --
def cpu_reference_rate(system, steps, threads, warmup=1):
    """Seconds per step of the reference's own step code on the host cores
    (oracle/_ref: Engine.cu kernels + host neighbour list), with its list
    update (every 200 steps, Constants.cuh:71) amortised: `warmup` untimed
    steps, then `steps` timed ones, and one timed list update."""
    from oracle import pyoracle as po
    if po.ref_available():
        ref = po.RefEngine(system, n_threads=threads)
        t0 = time.perf_counter()
        ref.update_nlists()
        t_nl = time.perf_counter() - t0
        if warmup > 0:
            ref.step(warmup)
        t0 = time.perf_counter()
        ref.step(steps)
        t_step = (time.perf_counter() - t0) / steps
        ref.close()
        kind, used = "reference", threads
    else:   # the C restatement of the same path, single-threaded
        t0 = time.perf_counter()
        lists = po.ref_nlist(system, cells=False, ss_cap=1024)
        t_nl = time.perf_counter() - t0
        s = system
        for _ in range(warmup):
            s, _, _, _ = po.ref_step(s, lists)
        t0 = time.perf_counter()
        for _ in range(steps):
            s, _, _, _ = po.ref_step(s, lists)
        t_step = (time.perf_counter() - t0) / steps
        kind, used = "port", 1
    return t_step + t_nl / 200.0, t_step, t_nl, kind, used


def metric_name(workload):
    """The headline metric string, identical in both arms."""
    return f"ns/day, {workload}"


def workload_text(workload, spec, n, ws):
    """What the workload is, in the benchmark's terms and where it departs from them."""
    if workload != WORKLOAD:
        return workload
    return (f"{workload}: 16 chains x 64 (4 LJ types, harmonic bonds/angles, periodic dihedrals, one compound per "
            f"chain) + 31,000 single-site solvents = {n} particles, 10 nm cubic PBC box, dt 2 fs, Berendsen 300 K "
            f"tau 0.1 ps; solvent positions uniform conditioned on a 0.28 nm minimum separation (0.95 sigma_ij where "
            f"larger), sampled by hard-sphere Monte Carlo from a lattice instead of sequential rejection; LJ cut at "
            f"1.2 nm with a C2 potential switch from 1.0 nm (plain truncation drifts); Verlet list skin 0.1 nm, "
            f"rebuilt when a particle moved > skin/2")


def run_reference_arm(args, ws, rank):
    """The reference's own step code (Engine.cu built for the host, oracle/_ref)
    on all host threads, on the same seeded box as the GPU arm.  The box is
    packed by oracle/liblima_inputs.so (builder.cpp built for the host), so
    this arm loads no library of the product."""
    if rank != 0:
        return
    from quantom_b200 import systems as S
    spec = S.CONFIGS[args.workload]
    system = S.make_system(args.workload, seed=args.seed, packer_lib=ROOT / "oracle" / "liblima_inputs.so")
    threads = os.cpu_count() or 1
    steps, warmup = max(1, args.steps), max(0, args.warmup)
    per_step, t_step, t_nl, kind, used = cpu_reference_rate(system, steps, threads, warmup)
    v = ns_per_day(spec.dt, per_step * 1e3)
    sample = (f"{steps} timed steps (after {warmup} untimed) of the reference's step code on the same "
              f"{system.n_particles}-particle box, reference semantics, {used} host threads, plus one "
              f"neighbour-list update ({t_nl:.2f} s) amortised over its 200-step period")
    print(json.dumps({
        "impl": "reference", "metric": metric_name(args.workload), "value": v, "unit": "ns/day", "n_gpus": ws,
        "steps": steps, "warmup": warmup, "ms_per_step": per_step * 1e3, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded)",
        "config": {"workload": workload_text(args.workload, spec, system.n_particles, ws),
                   "particles": system.n_particles, "semantics": "reference", "dt_fs": spec.dt * 1e6,
                   "force_integrate_ms_per_step": t_step * 1e3, "nlist_update_ms": t_nl * 1e3},
        "cpu_baseline": {"value": v, "unit": "ns/day", "cores": used, "kind": kind, "sample": sample},
        "e2e": {"value": v, "unit": "ns/day", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }), flush=True)


# ------------------------------------------------------------------ ours --
def run_ours(args, ws, rank, local, pg):
    import torch
    from quantom_b200 import engine as E
    from quantom_b200 import systems as S

    dev = torch.device("cuda", local)
    torch.cuda.set_device(dev)
    spec = S.CONFIGS[args.workload]
    system = S.make_system(args.workload, seed=args.seed + rank)
    n = system.n_particles
    stream = torch.cuda.Stream(device=dev)
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device=dev)   # > 126 MB L2

    # ---- plain FP32 physics path (headline) -----------------------------
    eng = E.Engine(system, physics_params(E, spec, E.PRECISION_FP32, stream.cuda_stream, local))
    timed_steps(eng, stream, max(3, args.warmup), flush)
    barrier(pg)
    launches0 = eng.kernel_launches()
    rebuilds0 = eng.rebuild_count()
    with ClockSampler(local) as clk:
        time.sleep(0.2)
        with clk.window():
            ms = timed_steps(eng, stream, args.steps, flush)
    launches = eng.kernel_launches() - launches0
    steps_per_rebuild = args.steps / max(1, eng.rebuild_count() - rebuilds0)
    ms_step = max_over_ranks(ms / args.steps, pg, dev)
    clocks = clk.summary()
    prof = eng.profile_steps(200)
    warm = torch.empty(16, dtype=torch.float32, device=dev)   # "flush" that leaves the L2 warm
    n_warm = max(50, args.steps // 2)
    ms_warm = timed_steps(eng, stream, n_warm, warm) / n_warm
    eng.close()

    # ---- mixed precision, same protocol ------------------------------------
    engm = E.Engine(system, physics_params(E, spec, E.PRECISION_MIXED, stream.cuda_stream, local))
    timed_steps(engm, stream, max(3, args.warmup // 2), flush)
    ms_mixed = timed_steps(engm, stream, max(50, args.steps // 2), flush) / max(50, args.steps // 2)
    prof_m = engm.profile_steps(200)
    ms_mixed_warm = timed_steps(engm, stream, n_warm, warm) / n_warm
    engm.close()

    # ---- the reference's own semantics on the GPU, same workload ------------
    pr = E.default_params(box_len=spec.box_len, cutoff=spec.cutoff, dt=spec.dt, device=local)
    pr.stream = stream.cuda_stream
    engr = E.Engine(system, pr)
    timed_steps(engr, stream, 5, flush)
    ms_ref_sem = timed_steps(engr, stream, 50, flush) / 50
    engr.close()

    # ---- end to end through the public API from host arrays -----------------
    torch.cuda.synchronize(dev)
    barrier(pg)
    t0 = time.perf_counter()
    e2e = E.Engine(system, physics_params(E, spec, E.PRECISION_FP32, None, local))
    h2d = (system.compounds.nbytes + system.states.nbytes + system.solvents.nbytes + system.bridges.nbytes +
           system.forcefield.nbytes)
    # every step's FP64 energies come back through the frame log: the device
    # ring is copied to pinned host memory in stream order, so no step waits
    # for the host
    e2e.log_start(1, ring_frames=256, flags=0)
    t1 = time.perf_counter()
    e2e.step(args.steps)   # the API's N-step call (the reference's step loop)
    frames = e2e.log_read()
    t2 = time.perf_counter()
    assert len(frames["steps"]) == args.steps and np.isfinite(frames["energies"]).all()
    d2h = frames["energies"].nbytes + frames["logdata"].nbytes + frames["steps"].nbytes
    st, prev = e2e.compound_states()
    sol = e2e.solvents()
    d2h += st.nbytes + prev.nbytes + sol.nbytes
    t3 = time.perf_counter()
    e2e.close()   # teardown (device and pinned frees) is outside the timed region
    t_e2e = max_over_ranks(t3 - t0, pg, dev)
    e2e_split = {"create_upload_s": t1 - t0, "steps_and_frame_log_s": t2 - t1, "readback_s": t3 - t2,
                 "close_s_untimed": time.perf_counter() - t3}

    if rank != 0:
        return
    # ---- parameter gradients (config 3), cost relative to the forward loss ---
    grad = grad_study(E, S, device=local, fd=True, fp64_fd=True)
    grad = {k: grad[k] for k in ("workload", "n_steps", "checkpoint_every", "ms_forward_loss", "ms_grad",
                                 "grad_over_forward", "grad", "fd_fp64_oracle", "rel_err_vs_fd_fp64",
                                 "fd_fp64_host_s", "fd_fp32_gpu", "rel_err_vs_fd_fp32_gpu", "fd_fp32_gpu_h1e-3",
                                 "rel_err_vs_fd_fp32_gpu_h1e-3")}
    grad["fd_note"] = ("rel_err_vs_fd_fp64: against central differences of the FP64 oracle loss at the specified "
                       "step (1e-4 relative), the check the target names; the FP32 central differences of the "
                       "GPU loss beside it carry the FP32 trajectories' rounding noise")
    # ---- roofline of the dominant kernel (k_step: pairs + integration) -------
    # The pair terms are bound by the FP32 pipe: 32 FLOP per unique pair within
    # r_c (minimum image 9, r^2 5, rcp 1, s^6 3, scalar force 5, vector force 3,
    # accumulation on both sides 6), pairs = N (4/3) pi r_c^3 rho / 2.  The peak
    # is clock-derived (148 SMs x 128 FP32 lanes x 2 FLOP x 1.965 GHz): the
    # measured-peaks file holds HBM and bf16 figures only.  HBM is reported
    # beside it on the compulsory 80 B per particle (read position + velocity,
    # write position, velocity, force), and the ncu-measured DRAM traffic of one
    # launch against those compulsory bytes.
    peaks = measured_peaks()
    hbm = peaks.get("hbm_gbs")
    hbm_src = "measured (MEASURED_PEAKS.json hbm_gbs)"
    if not hbm:
        hbm, hbm_src = 6650.0, "fallback"
    rho = n / spec.box_len ** 3
    pairs = n * (4.0 / 3.0) * math.pi * spec.cutoff ** 3 * rho / 2.0
    t_pair = prof["pair"] * 1e-3
    flops_pair = pairs * FLOP_PER_PAIR
    tflops = flops_pair / t_pair / 1e12
    compulsory = 80.0 * n
    list_len = (4.0 / 3.0) * math.pi * (spec.cutoff + SKIN) ** 3 * rho    # expected Verlet-list entries
    id_bytes = 2.0 if n <= 65536 else 4.0    # the list's slot ids are 16-bit while the slots fit
    bytes_list = n * (80.0 + id_bytes * list_len)
    traffic = ncu_traffic("k_step", args.workload)
    roofline = {
        "kernel": "k_step", "bound": "fp32", "achieved": tflops, "peak": FP32_NOMINAL_TFLOPS,
        "unit": "TFLOP/s", "frac": tflops / FP32_NOMINAL_TFLOPS, "traffic": traffic,
        "peak_source": "nominal, clock-derived (148 SMs x 128 lanes x 2 FLOP x 1.965 GHz); no measured FP32 figure",
        "kernel_ms": prof["pair"], "flops_per_launch": flops_pair, "unique_pairs_within_rc": pairs,
        "flop_per_pair": FLOP_PER_PAIR,
        "hbm": {"compulsory_bytes_per_launch": compulsory, "achieved_gbs": compulsory / t_pair / 1e9,
                "peak_gbs": hbm, "frac": compulsory / t_pair / 1e9 / hbm, "peak_source": hbm_src,
                "traffic_over_compulsory": (traffic / compulsory) if traffic else None,
                "list_inclusive": {"bytes_per_launch": bytes_list, "achieved_gbs": bytes_list / t_pair / 1e9,
                                   "frac": bytes_list / t_pair / 1e9 / hbm,
                                   "note": f"counts the {int(id_bytes)}-byte Verlet-list entries (an "
                                           "implementation choice, not algorithmic bytes)"}},
        "step": {"ms": ms_step, "frac_fp32": flops_pair / (ms_step * 1e-3) / 1e12 / FP32_NOMINAL_TFLOPS},
    }
    cpu = None
    c0 = None
    if ws == 1:
        per_step, t_step, t_nl, kind, used = cpu_reference_rate(system, args.cpu_sample_steps, os.cpu_count() or 1)
        cpu = {"value": ns_per_day(spec.dt, per_step * 1e3), "unit": "ns/day", "cores": used, "kind": kind,
               "sample": f"{args.cpu_sample_steps} steps of the same {n}-particle box through the reference's own "
                         f"Engine.cu step code (reference semantics) on {used} host threads, plus one neighbour-list "
                         f"update ({t_nl:.2f} s) amortised over its 200-step period",
               "force_integrate_ms_per_step": t_step * 1e3, "nlist_update_ms": t_nl * 1e3}
        c0 = c0_study(E, S, stream, flush, local)
    value = ws * ns_per_day(spec.dt, ms_step)
    out = {
        "metric": metric_name(args.workload), "value": value, "unit": "ns/day", "n_gpus": ws,
        "steps": args.steps, "warmup": max(3, args.warmup), "ms_per_step": ms_step, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded)",
        "mixed_ratio_to_fp32": ms_mixed / ms_step, "mixed_ms_per_step": ms_mixed,
        "gpu_launches": launches,
        "config": {"workload": workload_text(args.workload, spec, n, ws), "particles": n,
                   "semantics": "physics (conservative LJ + bonded forms, velocity Verlet), plain FP32",
                   "parallelism": f"replicas x{ws}" if ws > 1 else "single GPU",
                   "l2": "flushed before every timed step (256 MiB memset on the engine stream, outside the timed "
                         "events)"},
        "roofline": roofline,
        "e2e": {"value": ws * ns_per_day(spec.dt, t_e2e * 1e3 / args.steps), "unit": "ns/day",
                "h2d_bytes_per_step": h2d / args.steps, "d2h_bytes_per_step": d2h / args.steps,
                "split": e2e_split,
                "note": "engine created and box uploaded from host arrays inside the timed region, then one "
                        "N-step call; every step's FP64 energies read back through the frame log "
                        "(stream-ordered copies to pinned memory, no per-step sync), final state read back; the "
                        "engine's teardown comes after the clock stops"},
        "clocks": clocks,
        "mixed": {"ms_per_step": ms_mixed, "ratio_to_fp32": ms_mixed / ms_step,
                  "l2_warm": {"fp32_ms_per_step": ms_warm, "mixed_ms_per_step": ms_mixed_warm,
                              "ratio_to_fp32": ms_mixed_warm / ms_warm,
                              "note": "the same steps without the L2 flush in between"},
                  "ns_per_day": ns_per_day(spec.dt, ms_mixed), "kernels_ms": prof_m},
        "reference_semantics_gpu": {"ms_per_step": ms_ref_sem, "ns_per_day": ns_per_day(spec.dt, ms_ref_sem),
                                    "note": "the reference's own functional forms on the GPU, same box: the "
                                            "same-semantics counterpart of the CPU reference arm"},
        "kernels_ms": prof,
        "steps_per_list_rebuild": steps_per_rebuild,
        "grad": grad,
        "c0": c0,
    }
    if cpu:
        out["cpu_baseline"] = cpu
    print(json.dumps(out), flush=True)


def main():
    args = parse()
    if args.mode == "kernels":
        run_kernels_only(args)
        return
    if args.mode == "precision":
        run_precision(args)
        return
    if args.mode == "grad":
        run_grad(args)
        return
    if args.mode == "large":
        run_large(args)
        return
    if args.mode == "large-fp64":
        run_large_fp64(args)
        return
    if args.mode == "6lzm":
        run_6lzm(args)
        return
    ws, rank, local, pg = dist_setup(args) if args.impl == "ours" else (int(os.environ.get("WORLD_SIZE", "1")),
                                                                        int(os.environ.get("RANK", "0")), 0, None)
    try:
        if args.impl == "reference":
            run_reference_arm(args, ws, rank)
        else:
            run_ours(args, ws, rank, local, pg)
    finally:
        if pg is not None:
            pg.destroy_process_group()


if __name__ == "__main__":
    main()
