#!/usr/bin/env python
"""Benchmark of the DG-BGK pseudo-time sweep on B200.

One "step" is one pseudo-time step of the reference time loop (ADVNCE,
src/advnce.f90:220-449) over the whole case.  The default workload is the
supersonic channel: [-5,15]x[-5,5] as 200x100 quads (39 800 P1 triangles)
minus a unit-square obstacle, 24 x 48 velocities (1.3755e8 DOFs), Mach 2,
Kn 0.05, f stored in FP32 with FP64 moments and residual norms.  The metric
is DOF-updates/s = 3*NELEM*VNPNT*steps / device time of the time loop.
Beside it (one GPU): the reference's own test case tc1 timed per step (its
one published timing is 0.123 s per step on 160 MPI ranks), the plain FP64
path on the same workload, the large channel (400x200 quads, 32x64
velocities, 9.8e8 DOFs) per step, the time to steady state (L2 residual
1e-8) of eight warm-start-family channels plain FP64 vs batched FP32 with an
FP64 finish and extrapolation, cold and warm-started from a network trained
in the run, the end-to-end rate through the C ABI with host buffers, and the
oracle on the host cores.

Arms:
  --impl ours       : the sm_100a library through its C ABI.
  --impl reference  : the reference algorithm on the host cores (the oracle,
                      a C++ restatement of the Fortran: it cannot be compiled
                      here), FP32 like the shipped build, all host threads.

Multi-GPU (torchrun): the step does not shard in this build (velocity-space
sharding is future work), so N ranks run N independent replicas; value is
the aggregate DOF-updates/s over all ranks with the time taken as the max
over ranks.
"""
import argparse
import json
import os
import statistics
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(ROOT, "dg-bgk_b200"))

METRIC = "time-to-steady-state (res 1e-8) and DOF-updates/s: plain FP64 vs FP32+warm-start, 1 B200"
UNIT = "DOF-updates/s"


def args():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=40)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--config", default="channel", choices=["channel", "cavity", "large"])
    ap.add_argument("--precision", type=int, default=32, choices=[32, 64])
    ap.add_argument("--no-fp64", action="store_true", help="skip the plain-FP64 comparison leg")
    ap.add_argument("--no-cpu", action="store_true", help="skip the CPU baseline sample")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-steady", action="store_true", help="skip the time-to-steady-state leg")
    ap.add_argument("--no-tc1", action="store_true", help="skip the reference test case tc1 leg")
    ap.add_argument("--no-large", action="store_true", help="skip the large-channel (400x200, 32x64) leg")
    ap.add_argument("--no-cavity", action="store_true", help="skip the cavity's time to residual 1e-8")
    ap.add_argument("--shard", action="store_true",
                    help="velocity-space shards: the workload's speed rings split over the ranks (strong scaling, "
                         "NCCL all-reduces between the step's phases) instead of one replica per rank")
    return ap.parse_args()


def make_case(name):
    import dgbgk
    return {"channel": dgbgk.config2, "cavity": dgbgk.config1, "large": dgbgk.config5}[name]()


def workload(case, prec):
    m = case.mesh
    return (f"{case.name}: {m.nelem} P1 elements x {case.rorder}x{case.torder} velocities = {case.dofs} DOFs, "
            f"Mach {case.info.get('mach')}, Kn {case.info.get('kn')}, f in FP{prec}")


def config_of(case, prec, world):
    """The workload description both arms print (the same keys and values)."""
    sf = 4 if prec == 32 else 8
    return {"workload": workload(case, prec), "nelem": case.mesh.nelem, "vnpnt": case.rorder * case.torder,
            "dofs": case.dofs, "l2": f"inputs larger than L2: each f buffer is {case.dofs * sf / 1e6:.0f} MB",
            "parallelism": f"replicas x{world}" if world > 1 else "single GPU"}


# ------------------------------------------------------------------ dist ----
class Dist:
    def __init__(self):
        self.world = int(os.environ.get("WORLD_SIZE", "1"))
        self.rank = int(os.environ.get("RANK", "0"))
        self.local = int(os.environ.get("LOCAL_RANK", "0"))
        self.pg = None
        if self.world > 1:
            import datetime
            import torch
            import torch.distributed as dist
            backend = "nccl" if torch.cuda.is_available() else "gloo"
            if backend == "nccl":
                torch.cuda.set_device(self.local)
            dist.init_process_group(backend, timeout=datetime.timedelta(seconds=300))
            self.pg = dist
            self.backend = backend

    def barrier(self):
        if self.pg:
            self.pg.barrier()

    def max(self, x):
        if not self.pg:
            return x
        import torch
        dev = f"cuda:{self.local}" if self.backend == "nccl" else "cpu"
        t = torch.tensor([x], dtype=torch.float64, device=dev)
        self.pg.all_reduce(t, op=self.pg.ReduceOp.MAX)
        return float(t.item())

    def close(self):
        if self.pg:
            self.pg.destroy_process_group()


# ---------------------------------------------------------------- clocks ----
class Clocks:
    """SM clock and clock-event reasons sampled through NVML every ~2 ms in a
    thread during the timed region (the region can be a few tens of ms, too
    short for nvidia-smi's sampling); read-only queries."""

    REASONS = (("hw_slowdown", "nvmlClocksEventReasonHwSlowdown"),
               ("hw_thermal_slowdown", "nvmlClocksEventReasonHwThermalSlowdown"),
               ("sw_thermal_slowdown", "nvmlClocksEventReasonSwThermalSlowdown"),
               ("sw_power_cap", "nvmlClocksEventReasonSwPowerCap"))

    def __init__(self, cuda_index):
        self.cuda_index = cuda_index
        self.rows = []
        self.h = None
        self.nv = None
        self.run = False

    def _handle(self):
        import pynvml as nv
        import torch
        nv.nvmlInit()
        self.nv = nv
        try:
            uuid = str(torch.cuda.get_device_properties(self.cuda_index).uuid)
            return nv.nvmlDeviceGetHandleByUUID(uuid if uuid.startswith("GPU-") else "GPU-" + uuid)
        except Exception:
            return nv.nvmlDeviceGetHandleByIndex(self.cuda_index)

    def start(self):
        try:
            self.h = self._handle()
            self.max_mhz = float(self.nv.nvmlDeviceGetMaxClockInfo(self.h, self.nv.NVML_CLOCK_SM))
        except Exception:
            self.h = None
            return
        self.run = True
        self.th = threading.Thread(target=self._poll, daemon=True)
        self.th.start()

    def _poll(self):
        nv = self.nv
        while self.run:
            try:
                sm = float(nv.nvmlDeviceGetClockInfo(self.h, nv.NVML_CLOCK_SM))
                rs = int(nv.nvmlDeviceGetCurrentClocksEventReasons(self.h))
                self.rows.append((sm, rs))
            except Exception:
                break
            time.sleep(0.002)

    def stop(self):
        if self.h is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvml unavailable"], "samples": 0}
        self.run = False
        self.th.join(timeout=5)
        if not self.rows:
            return {"sm_mhz": None, "sm_max_mhz": self.max_mhz, "reasons": ["no samples"], "samples": 0}
        reasons = sorted({name for _, rs in self.rows for name, attr in self.REASONS
                          if rs & int(getattr(self.nv, attr, 0))})
        return {"sm_mhz": statistics.median(s for s, _ in self.rows), "sm_max_mhz": self.max_mhz,
                "reasons": reasons, "samples": len(self.rows), "source": "nvml"}


def peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        d = json.load(open(p))
        return float(d["hbm_gbs"]), "MEASURED_PEAKS.json hbm_gbs (of measured)"
    return 6650.0, "profiling-recipe fallback 6.65 TB/s (of fallback)"


def ncu_traffic(case_name, prec):
    """dram bytes per sweep launch from the committed ncu summary, if it
    covers this workload."""
    p = os.path.join(ROOT, "profiles", "sweep_traffic.json")
    if not os.path.exists(p):
        return None
    d = json.load(open(p))
    e = d.get(f"{case_name}/fp{prec}")
    return None if e is None else e.get("dram_bytes_per_launch")


def cpu_threads():
    try:
        return len(os.sched_getaffinity(0))
    except Exception:
        return os.cpu_count() or 1


def oracle_step_rate(case, nsteps, threads, warmup=0, min_seconds=0.0):
    """DOF-updates/s of the oracle's time step on the host cores: nsteps
    steps, or (min_seconds > 0) one timed step and then as many more as
    bring the sample to about min_seconds.  Returns the rate, the seconds
    and the steps timed."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    from pyoracle import Oracle
    o = Oracle.from_case(case, prec=32, threads=threads)
    i = case.init
    o.inicon2(i["T1"], i["P1"], i["U0"], i["V0"])
    if warmup:
        o.advance(warmup)
    t = time.perf_counter()
    o.advance(nsteps)
    dt = time.perf_counter() - t
    if min_seconds > 0 and dt < min_seconds:
        more = max(1, int(min_seconds / max(dt / nsteps, 1e-9)) - nsteps)
        t = time.perf_counter()
        o.advance(more)
        dt += time.perf_counter() - t
        nsteps += more
    o.close()
    return case.dofs * nsteps / dt, dt, nsteps


# The reference's own test case tc1 (tc/tc1/reentry_test.con: 28 304 P1
# elements, Lobatto40 x 40 angles = 1.359e8 DOFs, ALPHA 0.9, IMMAT 1, the
# namelist's gas with the reference's defaults R 287, M 32, d 250e-12),
# built from the committed fixtures, and the one published timing of the
# reference: 0.123 s per pseudo-time step on 160 MPI ranks, FP32
# (tc/tc1/output over its 2000 steps).
TC1_PUBLISHED_S_PER_STEP = 0.123


def tc1_leg(device, steps=40, warmup=3):
    from dgbgk.formats import read_lobatto, read_plt
    from dgbgk.solver import Solver, setup_mesh, vspace
    g = os.path.join(ROOT, "tests", "golden")
    mesh = read_plt(os.path.join(g, "tc1_reentry.plt.gz"))
    n, eta, w = read_lobatto(os.path.join(g, "Lobatto40.txt"))
    nml = json.load(open(os.path.join(g, "kat.json")))["tc1_namelist"]
    f = lambda k: float(nml[k])
    to = int(nml["TORDER"])
    st = setup_mesh(mesh.intma, mesh.coord, mesh.bsido)
    vc, sw = vspace(n, to, eta, w)
    dofs = 3 * mesh.nelem * n * to
    out = {"case": f"tc1 reentry: {mesh.nelem} P1 elements x {n}x{to} velocities = {dofs} DOFs, ALPHA "
                   f"{nml['ALPHA']}, IMMAT {nml['IMMAT']}", "dofs": dofs,
           "published_reference_s_per_step": TC1_PUBLISHED_S_PER_STEP,
           "published_reference_setup": "160 MPI ranks (16 space x 10 velocity partitions), FP32"}
    for prec in (32, 64):
        s = Solver(mesh.intma, mesh.coord, mesh.bsido, st, vc, sw, n, to, f("rv"), immat=int(nml["IMMAT"]),
                   csafm=f("CSAFM"), alpha=f("ALPHA"), rgas=287.0, molar_mass=32.0, diameter=250e-12,
                   cinf=(f("CINF(1)"), f("CINF(2)"), f("CINF(3)"), f("CINF(4)")), precision=prec, device=device)
        s.inicon2(f("T1"), f("P1"), f("U0"), f("V0"))
        s.advance(warmup)
        s.advance(steps)
        ms = s.last_ms() / steps
        out[f"fp{prec}"] = {"ms_per_step": ms, "dof_updates_per_s": dofs / (ms * 1e-3),
                            "speedup_vs_published": TC1_PUBLISHED_S_PER_STEP / (ms * 1e-3)}
        del s
    return out


def large_leg(device, steps=10, warmup=3):
    """The large channel ([-10,30]x[-10,10], 400x200 quads, 32x64
    velocities, 9.8e8 DOFs, Mach 1.5, Kn 0.02): ms per step and the kernels'
    achieved bandwidth at FP32 and FP64 (the time to steady state of this
    workload is recorded by dgbgk.steady, not here)."""
    from dgbgk import Solver, config5
    case = config5()
    names = ["k_moments", "k_wall", "k_sweep", "k_resid"]
    peak, _ = peaks()
    out = {"workload": workload(case, 32).replace(", f in FP32", ""), "dofs": case.dofs}
    for prec in (32, 64):
        sf = 4 if prec == 32 else 8
        s = Solver.from_case(case, precision=prec, device=device)
        s.init_case()
        s.advance(warmup)
        s.advance(steps)
        ms = s.last_ms() / steps
        k = s.profile(3)
        out[f"fp{prec}"] = {"ms_per_step": ms, "dof_updates_per_s": case.dofs / (ms * 1e-3),
                            "sweep_gbs": 2 * sf * case.dofs / (k[2] * 1e-3) / 1e9,
                            "sweep_frac": 2 * sf * case.dofs / (k[2] * 1e-3) / 1e9 / peak,
                            "moments_gbs": sf * case.dofs / (k[0] * 1e-3) / 1e9,
                            "kernel_ms": dict(zip(names, [float(x) for x in k]))}
        s.close()
    return out


def cavity_leg(device, tol=1e-8):
    """The 32 x 32 cavity with 16 x 32 velocities to residual tol: steps,
    device seconds and (FP32) the nodal fields' error against FP64's."""
    from dgbgk import config1
    import numpy as np
    from dgbgk import Solver
    from dgbgk.steady import march
    case = config1()
    out = {"workload": workload(case, 64).replace(", f in FP64", ""), "tol": tol}
    fields = {}
    ref = None
    for prec in (64, 32):
        s = Solver.from_case(case, precision=prec, device=device)
        s.init_case()
        r = march(s, tol, 3000000, ref=ref)
        if prec == 64:
            ref = r["ref"]  # both precisions stop at the same absolute residual
        m = s.macros()
        fields[prec] = np.stack([m["nd"], m["u"], m["v"], m["temp"]])
        out[f"fp{prec}"] = {"steps": r["steps"], "device_s": r["device_s"], "res_rel": r["res_rel"],
                            "converged": r["converged"]}
        s.close()
    vs = float(np.sqrt(case.rgas * case.init["T1"]))  # velocities on the thermal-speed scale
    a, b = fields[32], fields[64]
    out["fp32_rel_l2_vs_fp64"] = {k: float(np.linalg.norm(a[i] - b[i]) / max(np.linalg.norm(b[i]),
                                                                             vs * np.sqrt(b[i].size) if k in "uv" else 0.0))
                                  for i, k in enumerate(("n", "u", "v", "T"))}
    out["fp32_speedup"] = out["fp64"]["device_s"] / out["fp32"]["device_s"]
    return out


# ------------------------------------------------------------- our arm ----
def run_ours(a, d):
    import numpy as np
    import torch
    from dgbgk import Solver

    torch.cuda.set_device(d.local)
    case = make_case(a.config)
    s = Solver.from_case(case, precision=a.precision, device=d.local)
    s.init_case()
    s.advance(max(a.warmup, 3))
    info = s.info()
    clocks = Clocks(d.local)
    d.barrier()
    torch.cuda.synchronize()
    clocks.start()
    r = s.advance(a.steps)
    torch.cuda.synchronize()
    ck = clocks.stop()
    d.barrier()
    t_ms = d.max(s.last_ms())
    assert r["steps"] == a.steps
    dof_rate = d.world * case.dofs * a.steps / (t_ms * 1e-3)

    # dominant kernel, timed live with CUDA events on the library's stream
    kms = s.profile(5)
    names = ["k_moments", "k_wall", "k_sweep", "k_resid"]
    sf = 4 if a.precision == 32 else 8
    alg_bytes = 2 * sf * case.dofs  # one read + one write of f per DOF-update
    peak, peak_src = peaks()
    achieved = alg_bytes / (kms[2] * 1e-3) / 1e9
    traffic = ncu_traffic(case.name, a.precision)
    step_gbs = dof_rate / d.world * 2 * sf / 1e9

    out = {"metric": METRIC, "value": dof_rate, "unit": UNIT, "n_gpus": d.world, "steps": a.steps,
           "warmup": a.warmup, "ms_per_step": t_ms / a.steps, "higher_is_better": True,
           "scaling": "weak", "vs_baseline": None, "dtype": "f32" if a.precision == 32 else "f64",
           "data": "synthetic (generated mesh and velocity grid; free-stream initial state)",
           "config": config_of(case, a.precision, d.world),
           "launch": {"tile_elems": info["tile_elems"], "max_halo": info["max_halo"]},
           "roofline": {"bound": "hbm", "kernel": "k_sweep", "achieved": achieved, "peak": peak, "unit": "GB/s",
                        "frac": achieved / peak, "traffic": traffic, "peak_source": peak_src,
                        "alg_bytes_per_launch": alg_bytes,
                        "kernel_ms": dict(zip(names, [float(x) for x in kms])),
                        "step_frac": step_gbs / peak},
           "clocks": ck,
           "gpu_launches": a.steps * (4 if (case.mesh.bsido[:, 3] == 4).any() else 3)}
    del s
    # plain FP64 path on the same workload
    if not a.no_fp64 and a.precision == 32:
        s64 = Solver.from_case(case, precision=64, device=d.local)
        s64.init_case()
        s64.advance(max(a.warmup, 3))
        d.barrier()
        r64 = s64.advance(a.steps)
        t64 = d.max(s64.last_ms())
        k64 = s64.profile(3)
        out["fp64"] = {"value": d.world * case.dofs * a.steps / (t64 * 1e-3), "ms_per_step": t64 / a.steps,
                       "sweep_gbs": 16 * case.dofs / (k64[2] * 1e-3) / 1e9,
                       "kernel_ms": dict(zip(names, [float(x) for x in k64]))}
        out["fp32_over_fp64_per_step"] = out["value"] / out["fp64"]["value"]
        del s64
    # time to steady state (L2 residual 1e-8 of a cold start's first step)
    # on eight channels of the warm-start family: plain FP64 one case at a
    # time (the reference method); FP32 in one batch until 1e-5 (or its
    # rounding plateau), then FP64 to 1e-8 (the precision handoff), with
    # reduced-rank extrapolation of the iterates, from the cold start and
    # from the warm-start network's prediction.  The network (3 -> 256 x 3
    # -> 32768, BF16 tcgen05 GEMMs accumulating in FP32) is trained here by
    # the library's kernels on a training set this run generates: 48
    # channels of the same family (another seed) marched in FP32 batches to
    # 1e-4 of their first step's residual.  A case whose n, u or T ends more
    # than 1e-6 (relative L2) from the plain march's counts as a failure.
    if not a.no_steady and d.world == 1:
        from dgbgk.study import WarmStart, draw_cases, evaluate, generate
        t0 = time.perf_counter()
        X, Y, keep = generate(draw_cases(48, 78), tol=1e-4, accept=1e-3, device=d.local)
        gen_s = time.perf_counter() - t0
        ws = WarmStart(width=256, depth=3, batch=128, seed=0)
        hist = ws.fit(X, Y, schedule=((2000, 1e-3), (1000, 3e-4)))
        cases = draw_cases(8, 77)
        res, _, kept = evaluate(cases, ws, ways=("plain", "fast_cold_rre", "fast_rre"), device=d.local)
        st = {"cases": f"{len(kept)} channels [-5,15]x[-10,10], 100x100 quads, 16x32 velocities, free-stream "
                       "sides, Mach/Kn/obstacle drawn (dgbgk.study.draw_cases(8, 77))",
              "dofs_per_case": kept[0].dofs if kept else 0, "tol": 1e-8, "switch_tol": res["switch_tol"],
              "plain_fp64_s": res["plain"]["wall_s"], "plain_fp64_steps": int(sum(res["plain"]["steps"])),
              "batch_shapes": res.get("batch_shapes"),
              "timing": "wall seconds of each march from its initial state to tol (the plain arm one case after "
                        "another); the batch shape is tuned once per precision beforehand, untimed",
              "warm_start": {"network": "3 -> 256 x 3 -> 32768 (n, u, v, T on 64 x 128), BF16 tcgen05 GEMMs, FP32 "
                                        "accumulation, Adam", "train_cases": len(keep),
                             "train_cases_drawn": "dgbgk.study.draw_cases(48, 78), FP32 batches to 1e-4",
                             "generate_s": gen_s, "train_s": ws.train_s, "loss_first": float(hist[:10].mean()),
                             "loss_last": float(hist[-50:].mean())}}
        for k, name in (("fast_cold_rre", "fast_cold_rre"), ("fast_rre", "fast_warm_rre")):
            e = res[k]["rel_l2_vs_plain"]
            st[name] = {"wall_s": res[k]["wall_s"], "device_s": res[k]["device_s"],
                        "speedup_vs_plain": res[k]["speedup_vs_plain"],
                        "steps": int(sum(res[k]["steps"])), "steps_fp64_finish": int(sum(res[k]["steps_fp64_finish"])),
                        "max_rel_l2_vs_plain": res[k]["max_rel_l2_vs_plain"],
                        "cases_over_1e-6": int(sum(max(x["n"], x["u"], x["T"]) > 1e-6 for x in e)),
                        "fell_back_to_cold": res[k]["fell_back_to_cold"]}
        out["steady_state"] = st
    if not a.no_tc1 and d.world == 1:
        out["reference_case_tc1"] = tc1_leg(d.local)
    if not a.no_large and d.world == 1:
        out["large_channel"] = large_leg(d.local)
    # the lid-driven cavity (32 x 32 quads, 16 x 32 velocities, lid Mach
    # 0.3, Kn 0.1, seeded 1e-3 density perturbation) marched from its cold
    # start to L2 residual 1e-8 of its first step's, FP64 and FP32 f
    if not a.no_cavity and d.world == 1:
        out["cavity_steady"] = cavity_leg(d.local)
    # end to end through the C ABI with host buffers
    if not a.no_e2e:
        s = Solver.from_case(case, precision=a.precision, device=d.local)
        s.init_case()
        host = torch.empty((case.mesh.nelem, case.rorder * case.torder, 3),
                           dtype=torch.float32 if a.precision == 32 else torch.float64).pin_memory()
        hv = host.numpy()
        s.get_state(out=hv)
        s.advance(2)
        d.barrier()
        t0 = time.perf_counter()
        s.set_state(hv)         # H2D of DISNF(3,V,E) from the pinned buffer + layout change
        s.advance(a.steps)
        s.get_state(out=hv)     # layout change + D2H of the advanced DISNF into the pinned buffer
        t1 = time.perf_counter()
        te = d.max(t1 - t0)
        nb = host.numel() * host.element_size()
        out["e2e"] = {"value": d.world * case.dofs * a.steps / te, "unit": UNIT,
                      "h2d_bytes_per_step": nb / a.steps, "d2h_bytes_per_step": nb / a.steps,
                      "note": f"set_state + advance({a.steps}) + get_state per call, pinned host DISNF"}
        del s
    if d.rank == 0 and d.world == 1 and not a.no_cpu:
        thr = cpu_threads()
        rate, secs, n = oracle_step_rate(case, 1, thr, min_seconds=15.0)
        out["cpu_baseline"] = {"value": rate, "unit": UNIT, "cores": thr, "kind": "port",
                               "sample": f"{n} full pseudo-time steps of {case.name} (FP32, {secs:.1f} s, "
                                         f"{thr} OpenMP threads)"}
    return out


def run_sharded(a, d):
    """The workload split into whole speed rings over the ranks (one shard
    per GPU, dgbgk.shard): a step is the library's four phases with three
    all-reduces (NCCL, on the library's stream) between them; the time is
    the max over the ranks of the device time of the timed steps."""
    import torch
    from dgbgk.shard import ShardedSolver, TorchGroup, advance_distributed, advance_local
    torch.cuda.set_device(d.local)
    case = make_case(a.config)
    sh = ShardedSolver(case, d.rank, d.world, precision=a.precision, device=d.local)
    sh.init_case()

    def run(n):
        if d.world > 1:
            return advance_distributed(sh, n, group=TorchGroup(d.pg), poll_every=0)
        return advance_local([sh], n, poll_every=0)[0]
    run(max(a.warmup, 3))
    clocks = Clocks(d.local)
    d.barrier()
    torch.cuda.synchronize()
    clocks.start()
    r = run(a.steps)
    torch.cuda.synchronize()
    ck = clocks.stop()
    d.barrier()
    t_ms = d.max(sh.solver.last_ms())
    assert r["steps"] == a.steps
    rate = case.dofs * a.steps / (t_ms * 1e-3)  # the whole case advanced by all ranks together
    sh.close()
    return {"metric": METRIC, "value": rate, "unit": UNIT, "n_gpus": d.world, "steps": a.steps,
            "warmup": a.warmup, "ms_per_step": t_ms / a.steps, "higher_is_better": True, "scaling": "strong",
            "vs_baseline": None, "dtype": "f32" if a.precision == 32 else "f64",
            "data": "synthetic (generated mesh and velocity grid; free-stream initial state)",
            "config": dict(config_of(case, a.precision, 1),
                           parallelism=f"velocity shards x{d.world} (whole speed rings per GPU)"),
            "clocks": ck, "gpu_launches": a.steps * 7}


def run_reference(a, d):
    if d.rank != 0:
        return None
    case = make_case(a.config)
    thr = cpu_threads()
    rate, secs, _ = oracle_step_rate(case, a.steps, thr, warmup=a.warmup)
    return {"impl": "reference", "metric": METRIC, "value": rate, "unit": UNIT, "n_gpus": d.world,
            "steps": a.steps, "warmup": a.warmup, "ms_per_step": secs * 1e3 / a.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic (generated mesh and velocity grid; free-stream initial state)",
            "config": config_of(case, 32, d.world),
            "cpu_baseline": {"value": rate, "unit": UNIT, "cores": thr, "kind": "port",
                             "sample": f"{a.steps} full pseudo-time steps of {case.name} after {a.warmup} warm-up "
                                       f"steps (FP32, {thr} OpenMP threads)"},
            "e2e": {"value": rate, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}


def main():
    a = args()
    d = Dist()
    try:
        if a.impl == "reference":
            out = run_reference(a, d)
        elif a.shard:
            out = run_sharded(a, d)
        else:
            out = run_ours(a, d)
        if d.rank == 0 and out is not None:
            print(json.dumps(out), flush=True)
    finally:
        d.close()


if __name__ == "__main__":
    main()
