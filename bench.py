"""Benchmark of the B200 particle solver (prints one JSON line on rank 0).

python bench.py [--gpus N] [--steps K] [--warmup W] [--impl pfsim|reference]
                [--workload sort]

Under torchrun (N > 1) each rank drives one GPU; work is sharded by
independent units (scenes / sorts) with no data-path collective, timings are
taken with CUDA events on the launching stream and the max over ranks is
reported. `--impl reference` times the CPU restatement of the reference
algorithm (the oracle) on this host's cores instead.
"""

from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import time
from pathlib import Path

ROOT = Path(__file__).resolve().parent
PKG = ROOT / "threejs-particle-fluids_b200"
for _p in (str(ROOT), str(PKG)):
    if _p not in sys.path:
        sys.path.insert(0, _p)

import numpy as np  # noqa: E402

PEAKS_FILE = ROOT / "MEASURED_PEAKS.json"
FALLBACK_HBM_GBS = 6650.0


def hbm_peak() -> tuple[float, str]:
    try:
        d = json.loads(PEAKS_FILE.read_text())
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return FALLBACK_HBM_GBS, "fallback"


# ------------------------------------------------------------ clocks ----
class ClockSampler:
    """nvidia-smi clock/throttle samples during the timed region."""

    FIELDS = (
        "index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
        "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
        "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap"
    )

    def __init__(self, device: int):
        self.device = device
        self.proc = None

    def start(self):
        """Starts sampling and returns once the first sample is out, so that
        nvidia-smi's own start-up (NVML initialisation, which can hold up the
        driver for tens of milliseconds) is over before the timed region."""
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.device), f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits", "-lms", "100"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True,
            )
        except Exception:
            self.proc = None
            return
        import select

        ready, _, _ = select.select([self.proc.stdout], [], [], 10.0)
        if ready:
            self.proc.stdout.readline()  # taken before the timed region: not counted

    def stop(self) -> dict:
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        time.sleep(0.25)
        self.proc.terminate()
        try:
            out, _ = self.proc.communicate(timeout=5)
        except Exception:
            self.proc.kill()
            out = ""
        sm, smax, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in out.strip().splitlines():
            parts = [p.strip() for p in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                smax.append(float(parts[2]))
            except ValueError:
                continue
            for nm, v in zip(names, parts[5:9]):
                if v.lower() == "active":
                    reasons.add(nm)
        return {
            "sm_mhz": statistics.median(sm) if sm else None,
            "sm_max_mhz": max(smax) if smax else None,
            "reasons": sorted(reasons),
            "samples": len(sm),
        }


# --------------------------------------------------------- workloads ----
class SortWorkload:
    """Standalone hash-grid counting sort, 16M float4 positions on a 128^3
    linear grid (uniform distribution); one step = one stable sort."""

    name = "grid_sort_16M_uniform_128cubed"
    metric = "particles sorted/s"
    unit = "particles/s"

    def __init__(self, n: int = 16_000_000, dist: str = "uniform"):
        self.n = n
        self.dist = dist
        self.cells = 128**3

    def host_input(self, seed: int) -> np.ndarray:
        from pfsim import workloads as W

        return W.sort_uniform(self.n, seed) if self.dist == "uniform" else W.sort_blobs(self.n, seed)

    # DRAM bytes per particle of one sort of this workload (uniform), the sum
    # of dram__bytes_read.sum + dram__bytes_write.sum over a sort's launches
    # from a one-pass ncu capture:
    #   ncu --metrics gpu__time_duration.sum,dram__bytes_read.sum,
    #       dram__bytes_write.sum --clock-control none -s 40 -c 60 --csv
    #       python bench.py --workload sort --steps 3 --warmup 3
    #       --no-cpu-baseline
    TRAFFIC_PER_PARTICLE = 63.4

    def launches(self) -> int:
        """Kernel launches of one sort: keys with digit counts, digit starts,
        per radix pass (digits of at most 8 bits) tile counts, two tile-count
        scans and the scatter, then the start scan."""
        bits = max(1, (self.cells - 1).bit_length())
        return 2 + 4 * -(-bits // 8) + 1

    def algorithmic_bytes(self) -> int:
        # read x (16 B) + write perm (4 B) per particle; start + count (8 B) per cell
        return 20 * self.n + 8 * self.cells

    def grid(self):
        from pfsim import hashgrid as H
        from pfsim import workloads as W

        return H.GridOptions(cell_size=W.SORT_CELL, kind="linear", dims=W.SORT_GRID_DIMS)

    def run_gpu(self, steps: int, warmup: int, rank: int, world: int, dist_barrier) -> dict:
        import ctypes as C

        import torch

        from pfsim import _native as N

        L = N.lib()
        dev = torch.device("cuda", torch.cuda.current_device())
        host = self.host_input(1000 + rank)
        pos = torch.from_numpy(host).to(dev)
        perm = torch.empty(self.n, dtype=torch.int32, device=dev)
        start = torch.empty(self.cells, dtype=torch.int32, device=dev)
        count = torch.empty(self.cells, dtype=torch.int32, device=dev)
        desc = self.grid().desc(self.n)
        stream = torch.cuda.current_stream(dev)
        sp = C.c_void_p(stream.cuda_stream)

        def one():
            N.check(L.pf_sort(C.c_void_p(pos.data_ptr()), self.n, C.byref(desc), C.c_void_p(perm.data_ptr()),
                              C.c_void_p(start.data_ptr()), C.c_void_p(count.data_ptr()), None, None, sp))

        for _ in range(warmup):
            one()
        torch.cuda.synchronize()
        dist_barrier()
        torch.cuda.synchronize()
        clocks = ClockSampler(dev.index)
        clocks.start()
        ev0 = torch.cuda.Event(enable_timing=True)
        ev1 = torch.cuda.Event(enable_timing=True)
        ev0.record(stream)
        for _ in range(steps):
            one()
        ev1.record(stream)
        torch.cuda.synchronize()
        dist_barrier()
        ms = ev0.elapsed_time(ev1) / steps
        clk = clocks.stop()
        err = C.c_uint32(0)
        N.check(L.pf_sort_device_errors(sp, C.byref(err)))
        if err.value:
            raise RuntimeError(f"device error word {err.value}")

        # End to end through the host-buffer C ABI (H2D of positions and D2H of
        # perm, start and count inside the timed region), pinned host memory.
        h_pos = torch.from_numpy(host).pin_memory()
        h_perm = torch.empty(self.n, dtype=torch.int32).pin_memory()
        h_start = torch.empty(self.cells, dtype=torch.int32).pin_memory()
        h_count = torch.empty(self.cells, dtype=torch.int32).pin_memory()
        u32 = C.POINTER(C.c_uint32)

        def one_host():
            N.check(L.pf_sort_host(C.cast(C.c_void_p(h_pos.data_ptr()), C.POINTER(C.c_float)), self.n, C.byref(desc),
                                   C.cast(C.c_void_p(h_perm.data_ptr()), u32), C.cast(C.c_void_p(h_start.data_ptr()), u32),
                                   C.cast(C.c_void_p(h_count.data_ptr()), u32), None, None))

        for _ in range(max(1, warmup)):
            one_host()
        e_steps = max(3, steps // 2)
        legacy = torch.cuda.default_stream(dev)
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        e0.record(legacy)
        for _ in range(e_steps):
            one_host()
        e1.record(legacy)
        torch.cuda.synchronize()
        e2e_ms = e0.elapsed_time(e1) / e_steps
        return {
            "ms": ms,
            "units_per_step": self.n,
            "kernel_ms": ms,
            "kernel_name": "grid sort pipeline (keys with digit counts, digit starts, LSD radix passes of "
                           "tile counts + two tile-count scans + scatter, the last also counting the cells, "
                           "start scan)",
            "algorithmic_bytes": self.algorithmic_bytes(),
            "traffic": self.TRAFFIC_PER_PARTICLE * self.n if self.dist == "uniform" else None,
            "gpu_launches_per_step": self.launches(),
            "clocks": clk,
            "e2e_ms": e2e_ms,
            "h2d": 16 * self.n,
            "d2h": 4 * self.n + 8 * self.cells,
        }

    def run_cpu(self, threads: int) -> dict:
        from oracle import oracle as O

        O.set_threads(threads)
        host = self.host_input(1000)
        desc = self.grid().desc(self.n)
        O.sort(host[:1000], desc)
        t0 = time.perf_counter()
        reps = 0
        while True:
            O.sort(host, desc)
            reps += 1
            if time.perf_counter() - t0 > 3.0 or reps >= 3:
                break
        s = (time.perf_counter() - t0) / reps
        return {"seconds_per_step": s, "units_per_step": self.n, "reps": reps,
                "sample": f"{reps} full {self.n}-particle stable counting sorts", "cores": 1}


class BatchWorkload:
    """Batched solver over 256 uneven scenes: particle counts log-uniform on
    [5k, 200k], 70% dam-break fluids (container scale U[0.5, 2]) and 30% cloth
    sheets of 64^2-256^2 particles, 2 substeps x 4 iterations, dt = 1/60.
    One step = one frame of every scene. The same scenes are also stepped the
    plain way (each scene its own stream and launches, no graph) as the
    baseline of the batched/plain ratio."""

    name = "batch_256_scenes_5k-200k_fluid70_cloth30_S2_I4"
    metric = "particle-substeps/s & p99 step latency: batched/served vs plain, 1\u00d7B200"
    unit = "particle-substeps/s"
    DT = 1.0 / 60.0
    # The fluid neighbour stages, as pf_batch_profile_stage numbers them, with
    # their compulsory bytes per fluid particle in these single-fluid scenes of
    # one mass (neighbour gathers served on chip, the list itself excluded):
    #   0 list build (+ the first iteration's density and lambda): x* in;
    #     density and the (x*, lambda) record out = 16 + 4 + 16
    #   1 density + lambda: x* in; density and (x*, lambda) out = 36
    #   2 position correction with the apply fused: (x*, lambda) in, x* out
    #     and the collider test's committed position read on contact = 36
    #   3 XSPH: x and v in, the velocity change out = 48
    STAGES = {0: ("list build + first density", 36), 1: ("density + lambda", 36),
              2: ("position correction + apply", 36), 3: ("XSPH", 48)}
    # DRAM bytes per fluid particle of one launch of a stage, from a one-pass
    # ncu capture (dram__bytes_read.sum + dram__bytes_write.sum) of that
    # stage's pf_batch_profile_stage launches on this workload at the frame the
    # bench profiles it (after 3 warm-up and 20 timed frames; mean of 11
    # launches, 9,441,833 fluid particles), taken with
    #   ncu --nvtx --nvtx-include "stage_profile/" --metrics dram__bytes_read.sum,
    #       dram__bytes_write.sum,gpu__time_duration.sum --clock-control none
    #       -k regex:k_s_ -c 44 --csv python bench.py --steps 20 --warmup 3
    #       --no-cpu-baseline --no-plain --no-serve
    # (PFSIM_NBR_WIDE=0 or 1 fixes the list entry width the autotuner would
    # pick, for the figures of the other width). Keyed by that width in bits.
    STAGE_TRAFFIC_PER_PARTICLE: dict[int, dict[int, float]] = {
        16: {0: 151.1, 1: 127.6, 2: 168.9, 3: 140.0},
        32: {0: 286.6, 1: 207.6, 2: 248.8, 3: 216.1},
    }

    def __init__(self, n_scenes: int = 256):
        self.n_scenes = n_scenes

    def recipes(self, seed: int):
        from pfsim import workloads as W

        return W.batch_stream(self.n_scenes, seed=seed)

    def run_gpu(self, steps: int, warmup: int, rank: int, world: int, dist_barrier, plain_baseline=True) -> dict:
        import ctypes as C

        import torch

        from pfsim import _native as N
        from pfsim import recipe as R

        L = N.lib()
        backend = R.NativeBackend()
        recipes = self.recipes(replica_seed(rank))
        plain = [backend.build(r) for r in recipes]
        psub = sum(r.particle_substeps for r in recipes)
        # Both arms start from the scenes' initial state and are timed over
        # the same frames (after `warmup` frames): the batch copies the built
        # scenes' initial state, and the plain scenes are built afresh from
        # the same recipes once the batch is gone (each arm alone on the GPU).
        # ---- batched: one world, one launch per stage, one graph per tick
        batch = R.Batch(plain, use_graph=True)
        for sc in plain:
            sc.close()
        plain = None
        stream = torch.cuda.ExternalStream(L.pf_batch_stream(batch.h))
        for _ in range(warmup):
            batch.step(self.DT)
        torch.cuda.synchronize()
        dist_barrier()
        torch.cuda.synchronize()
        clocks = ClockSampler(torch.cuda.current_device())
        clocks.start()
        evs = [torch.cuda.Event(enable_timing=True) for _ in range(steps + 1)]
        torch.cuda.nvtx.range_push("timed_steps")  # an ncu launch list can select these launches
        evs[0].record(stream)
        for k in range(steps):
            batch.step(self.DT)
            evs[k + 1].record(stream)
        torch.cuda.synchronize()
        torch.cuda.nvtx.range_pop()
        dist_barrier()
        clk = clocks.stop()
        per = [evs[k].elapsed_time(evs[k + 1]) for k in range(steps)]
        ms = evs[0].elapsed_time(evs[-1]) / steps
        launches = int(L.pf_batch_launches_per_step(batch.h))
        # ---- the neighbour stages, event-timed on the batch stream on the
        # state the timed frames left (each launched 10 times after one
        # untimed launch); launches per step from the substeps and iterations
        sub = max(r.loop.substeps for r in recipes)
        its = max(r.loop.iterations for r in recipes)
        per_step = {0: sub, 1: sub * (its - 1), 2: sub * its, 3: sub}
        stages, items = {}, C.c_uint64(0)
        torch.cuda.nvtx.range_push("stage_profile")
        for sid in self.STAGES:
            st_ms = C.c_float(0)
            N.check(L.pf_batch_profile_stage(batch.h, sid, 10, C.byref(st_ms), C.byref(items)))
            stages[sid] = st_ms.value
        torch.cuda.nvtx.range_pop()
        tp, tb, tu, tg, te = (C.c_uint32(0) for _ in range(5))
        N.check(L.pf_batch_tuning(batch.h, C.byref(tp), C.byref(tb), C.byref(tu), C.byref(tg), C.byref(te)))
        # ---- end to end: per step the scene parameters go host->device (pinned)
        # and every scene's positions come back to pinned host memory. Each
        # step's read is asynchronous (as the reference's readback): its copy
        # runs beside the next step, into two pinned buffers in turn, and the
        # timed region ends after the last read has landed.
        total = sum(r.capacity for r in recipes)
        hosts = [torch.empty(total * 4, dtype=torch.float32).pin_memory() for _ in range(2)]
        hps = [C.cast(C.c_void_p(h.data_ptr()), C.POINTER(C.c_float)) for h in hosts]
        nbytes = hosts[0].numel() * 4
        e_steps = max(3, steps // 2)
        for k in range(2):
            batch.step(self.DT)
            N.check(L.pf_batch_read_positions_async(batch.h, hps[k & 1], nbytes))
        N.check(L.pf_batch_wait_reads(batch.h))
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        e0.record(stream)
        for k in range(e_steps):
            batch.step(self.DT)
            N.check(L.pf_batch_read_positions_async(batch.h, hps[k & 1], nbytes))
        N.check(L.pf_batch_wait_reads(batch.h))  # every step's positions are on the host
        e1.record(stream)
        torch.cuda.synchronize()
        e2e_ms = e0.elapsed_time(e1) / e_steps
        h2d = int(L.pf_batch_step_upload_bytes(batch.h))
        host = hosts[(e_steps - 1) & 1]
        ok = np.isfinite(host.numpy()).all()
        batch.close()
        if not ok:
            raise RuntimeError("non-finite positions after the timed steps")
        # ---- plain baseline: each scene its own launches and waits.
        # Sequential: step a scene and wait for it (the reference's
        # `await simulation.step()` per scene); timed as the sum of each
        # scene's device time between its step's start and end events.
        # Overlapped: every scene launched on its own stream, one wait.
        plain = [backend.build(r) for r in recipes] if plain_baseline else []
        for _ in range(warmup if plain_baseline else 0):
            for sc in plain:
                sc.step(self.DT)
        torch.cuda.synchronize()
        p_steps = max(2, steps) if plain_baseline else 0
        seq_dev = 0.0
        t0 = time.perf_counter()
        for _ in range(p_steps):
            for sc in plain:
                sc.step(self.DT)
                seq_dev += sc.last_step_ms()
        seq_wall = (time.perf_counter() - t0) * 1e3 / max(p_steps, 1)
        plain_ms = seq_dev / max(p_steps, 1) if plain_baseline else float("nan")
        o_steps = max(2, steps // 2) if plain_baseline else 0
        t0 = time.perf_counter()
        for _ in range(o_steps):
            for sc in plain:
                sc.step(self.DT)
        torch.cuda.synchronize()
        overlap_ms = (time.perf_counter() - t0) * 1e3 / max(o_steps, 1) if plain_baseline else float("nan")
        for sc in plain:
            sc.close()
        plain = None
        peak, _ = hbm_peak()
        table = {}
        traffic = self.STAGE_TRAFFIC_PER_PARTICLE.get(te.value, {})
        for sid, (label, bpp) in self.STAGES.items():
            gbs = bpp * items.value / (stages[sid] * 1e-3) / 1e9
            table[label] = {"ms_per_launch": stages[sid], "launches_per_step": per_step[sid],
                            "ms_per_step": stages[sid] * per_step[sid],
                            "share_of_step": stages[sid] * per_step[sid] / ms,
                            "bytes_per_fluid_particle": bpp, "achieved_gbs": gbs, "frac": gbs / peak,
                            "dram_bytes_per_fluid_particle": traffic.get(sid)}
        dom = max(self.STAGES, key=lambda sid: stages[sid] * per_step[sid])
        tpp = traffic.get(dom)
        return {
            "ms": ms,
            "units_per_step": psub,
            "kernel_ms": stages[dom],
            "kernel_name": self.STAGES[dom][0] + (" (warp-tile path)" if tp.value == 1 else " (slot path)"),
            "algorithmic_bytes": self.STAGES[dom][1] * items.value,
            # the captured figures are of the slot path
            "traffic": tpp * items.value if (tpp is not None and tp.value == 0) else None,
            "stages": table,
            "gpu_launches_per_step": launches,
            "clocks": clk,
            "e2e_ms": e2e_ms,
            "h2d": h2d,
            "d2h": 16 * total,
            "extra": {
                "p50_step_ms": float(np.percentile(per, 50)),
                "p99_step_ms": float(np.percentile(per, 99)),
                "plain_ms_per_step": plain_ms,
                "plain_value": psub / (plain_ms * 1e-3),
                "batched_over_plain": plain_ms / ms,
                "plain_wall_ms_per_step": seq_wall if plain_baseline else float("nan"),
                "plain_overlapped_ms_per_step": overlap_ms,
                "batched_over_plain_overlapped": overlap_ms / ms,
                "tuning": {"nbr_path": "tiles" if tp.value == 1 else "slots", "block": tb.value,
                           "fetch_depth": tu.value, "l2_group_particles": tg.value, "list_entry_bits": te.value},
                "scenes": len(recipes),
                "particles": total,
                "fluid_particles": int(items.value),
            },
        }

    def run_cpu(self, threads: int, budget_particles: int = 150_000, steps: int = 3) -> dict:
        """The oracle on a bounded sample of the same scene stream: the first
        scenes of the stream up to `budget_particles`, stepped `steps` frames."""
        from oracle import oracle as O

        recipes = self.recipes(1000)
        sample, n = [], 0
        for r in recipes:
            if n >= budget_particles:
                break
            sample.append(r)
            n += r.capacity
        be = O.OracleBackend(threads=threads)
        scenes = [be.build(r) for r in sample]
        for sc in scenes:
            sc.step(self.DT)
        t0 = time.perf_counter()
        for _ in range(steps):
            for sc in scenes:
                sc.step(self.DT)
        s = (time.perf_counter() - t0) / steps
        psub = sum(r.particle_substeps for r in sample)
        return {"seconds_per_step": s, "units_per_step": psub, "cores": threads,
                "sample": f"{len(sample)} scenes ({n} particles) of the same stream, {steps} frames each"}


class ServeWorkload:
    """Serving: a seeded Poisson stream of scene requests (N log-uniform on
    [5k, 500k], fluid/soft/cloth 60/20/20, lifetime U[60, 600] ticks), admitted
    under a 150 GB HBM budget and stepped every tick on device-resident
    state. The run starts from a steady-state population (`live` scenes with
    residual lifetimes) and keeps it by arrivals at live / mean lifetime per
    tick. The same stream is served twice: batched (cohorts, graphs) and
    plain (every scene its own world and stream)."""

    name = "serve_poisson_5k-500k_fluid60_soft20_cloth20_budget150GB"
    metric = BatchWorkload.metric
    unit = "particle-substeps/s"
    DT = 1.0 / 60.0
    MEAN_LIFE = 330.0

    def __init__(self, live: int = 96, seed: int = 7):
        self.live = live
        self.seed = seed

    def stream(self, ticks: int):
        """(tick, recipe, lifetime) in arrival order; tick 0 holds the
        initial population with residual lifetimes."""
        from pfsim import workloads as W

        r = W.rng(self.seed)
        out = []
        idx = 0
        for _ in range(self.live):
            rec, life = W.serve_request(r, idx, self.seed)
            rec.motion = None
            out.append((0, rec, max(1, int(r.integers(1, life + 1)))))
            idx += 1
        rate = self.live / self.MEAN_LIFE
        for t in range(1, ticks):
            for _ in range(int(r.poisson(rate))):
                rec, life = W.serve_request(r, idx, self.seed)
                rec.motion = None
                out.append((t, rec, life))
                idx += 1
        return out

    def serve(self, stream, ticks: int, warmup: int, plain: bool):
        import torch

        from pfsim import recipe as R

        srv = R.Server(budget_bytes=150 * 10**9, plain=plain, async_build=not plain, max_cohorts=4)
        by_tick = {}
        for t, rec, life in stream:
            by_tick.setdefault(t, []).append((rec, life))
        for rec, life in by_tick.get(0, []):
            srv.submit(rec, life)
        srv.tick(self.DT)  # admits the initial population (its cohort build starts)
        srv.drain()  # and waits for that build, so the run starts from a live population
        tick_ms, step_ms, ps0 = [], [], 0
        clocks = ClockSampler(torch.cuda.current_device())
        for t in range(warmup + ticks):
            if t == warmup:
                torch.cuda.synchronize()
                ps0 = srv.stats()["particle_substeps"]
                clocks.start()
                # an ncu launch list can select the timed ticks' launches
                torch.cuda.nvtx.range_push("plain_ticks" if plain else "served_ticks")
            for rec, life in by_tick.get(t + 1, []):
                srv.submit(rec, life)
            t0 = time.perf_counter()
            srv.tick(self.DT)
            if t >= warmup:
                ms = (time.perf_counter() - t0) * 1e3
                tick_ms.append(ms)
                # the tick without its admission: the plain server builds each
                # admitted request's world inside the tick, the batched one
                # only starts a cohort build there (it runs on a worker thread)
                step_ms.append(max(ms - srv.stats()["last_admit_ms"], 0.0))
        torch.cuda.nvtx.range_pop()
        clk = clocks.stop()
        st = srv.stats()
        srv.close()
        ps = st["particle_substeps"] - ps0
        wall, stepping = sum(tick_ms), sum(step_ms)
        return {"value": ps / (wall * 1e-3), "ms": wall / ticks, "p50": float(np.percentile(tick_ms, 50)),
                "p99": float(np.percentile(tick_ms, 99)), "clocks": clk, "stats": st,
                "ps_per_tick": ps / ticks, "step_value": ps / (stepping * 1e-3),
                "step_p50": float(np.percentile(step_ms, 50)), "step_p99": float(np.percentile(step_ms, 99))}

    def run_cpu(self, threads: int, budget_particles: int = 150_000, steps: int = 2) -> dict:
        """The oracle on the first requests of the same stream, up to
        `budget_particles`, stepped `steps` ticks."""
        from oracle import oracle as O

        sample, n = [], 0
        for _, rec, _ in self.stream(1):
            if n >= budget_particles:
                break
            sample.append(rec)
            n += rec.capacity
        be = O.OracleBackend(threads=threads)
        scenes = [be.build(r) for r in sample]
        for sc in scenes:
            sc.step(self.DT)
        t0 = time.perf_counter()
        for _ in range(steps):
            for sc in scenes:
                sc.step(self.DT)
        sec = (time.perf_counter() - t0) / steps
        return {"seconds_per_step": sec, "units_per_step": sum(r.particle_substeps for r in sample), "cores": threads,
                "sample": f"{len(sample)} requests ({n} particles) of the same stream, {steps} ticks"}

    def run_gpu(self, steps: int, warmup: int, rank: int, world: int, dist_barrier, plain_baseline=True) -> dict:
        stream = self.stream(warmup + steps + 1)
        b = self.serve(stream, steps, warmup, plain=False)
        p = self.serve(stream, steps, warmup, plain=True) if plain_baseline else None
        return {
            "ms": b["ms"], "units_per_step": b["ps_per_tick"], "clocks": b["clocks"],
            "extra": {
                "p50_tick_ms": b["p50"], "p99_tick_ms": b["p99"],
                # the plain arm without its world builds (a fair per-tick
                # stepping cost), and with them
                "plain_value": p["step_value"] if p else None,
                "plain_p50_tick_ms": p["step_p50"] if p else None,
                "plain_p99_tick_ms": p["step_p99"] if p else None,
                "served_over_plain": (b["value"] / p["step_value"]) if p else None,
                "plain_with_builds_value": p["value"] if p else None,
                "plain_with_builds_p99_tick_ms": p["p99"] if p else None,
                "requests": len(stream), "cohort_builds": b["stats"]["rebuilds"],
                "max_swap_ms": b["stats"]["max_swap_ms"], "max_admit_ms": b["stats"]["max_admit_ms"],
                "max_step_ms": b["stats"]["max_step_ms"], "max_free_ms": b["stats"]["max_free_ms"],
                "plain_max_admit_ms": p["stats"]["max_admit_ms"] if p else None,
                "live_at_end": b["stats"]["live"], "queued_at_end": b["stats"]["queued"],
            },
        }


class SceneWorkload:
    """One plain scene stepped through pf_step: `dam` is the 5,000-particle
    dam break (2 substeps x 4 iterations, XSPH 0.01), `mixed` the 50,000-particle
    fluid + 20 soft bodies + moving sphere scene (3 substeps x 4 iterations),
    `contacts` 50,000 particles of soft bodies (100 of ~500) piling up with
    particle contacts on (3 x 4), `cloth` a 256 x 256 sheet with stretch,
    bending and tether colours, drag and lift in a wind, and velocity
    smoothing (2 x 4)."""

    metric = "particle-substeps/s (one plain scene)"
    unit = "particle-substeps/s"
    DT = 1.0 / 60.0
    NAMES = {"dam": "dam_break_5k_S2_I4", "mixed": "mixed_50k_fluid30k_soft20x1k_sphere_S3_I4",
             "contacts": "softbody_pile_50k_contacts_S3_I4",
             "cloth": "cloth_256x256_bend_tether_aero_damping_S2_I4"}

    def __init__(self, which: str):
        self.which = which
        self.name = self.NAMES[which]

    def recipe(self):
        from pfsim import workloads as W

        if self.which == "dam":
            return W.dam_break(5000, seed=0)
        if self.which == "mixed":
            return W.mixed_scene(50_000, seed=0)
        if self.which == "contacts":
            r = W.softbody_pile(50_000, seed=0, per_body=500)
            r.loop.contact = True
            return r
        return W.cloth_sheet(256, seed=0, bend_compliance=1e-5, tethers=True, stretch_tolerance=0.06,
                             wind=(0.8, 0.0, 1.5), drag=0.18, lift=0.02, damping=0.1)

    def run_gpu(self, steps: int, warmup: int) -> dict:
        import torch

        from pfsim import _native as N
        from pfsim import recipe as R

        r = self.recipe()
        sc = R.NativeBackend().build(r)
        for _ in range(warmup):
            sc.step(self.DT)
        torch.cuda.synchronize()
        stream = torch.cuda.ExternalStream(N.lib().pf_scene_stream(sc.h))
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        clocks = ClockSampler(torch.cuda.current_device())
        clocks.start()
        e0.record(stream)
        for _ in range(steps):
            sc.step(self.DT)
        e1.record(stream)
        torch.cuda.synchronize()
        clk = clocks.stop()
        ms = e0.elapsed_time(e1) / steps
        return {"ms": ms, "value": r.particle_substeps / (ms * 1e-3), "clocks": clk, "particles": r.capacity}

    def run_cpu(self, threads: int, steps: int = 3) -> dict:
        from oracle import oracle as O

        r = self.recipe()
        sc = O.OracleBackend(threads=threads).build(r)
        sc.step(self.DT)
        t0 = time.perf_counter()
        for _ in range(steps):
            sc.step(self.DT)
        sec = (time.perf_counter() - t0) / steps
        return {"seconds_per_step": sec, "units_per_step": r.particle_substeps, "cores": threads,
                "sample": f"the same scene, {steps} frames after one warm-up frame"}


class MeshWorkload:
    """Mesh -> particle setup on the GPU: `bake` bakes a 64 x 64 UV sphere
    (3,968 triangles) into a 128^3 signed-distance grid (pf_bake_sdf);
    `voxelize` fills a 48 x 24 torus (2,304 triangles) with particles of
    radius 2.5 mm (pf_voxelize_mesh, about 1.9 M grid points). The unit is
    grid-point x triangle tests per second (the brute force both the
    reference and this build run)."""

    unit = "point-triangle tests/s"

    def __init__(self, which: str):
        self.which = which
        self.metric = {"bake": "SDF bake throughput", "voxelize": "voxeliser throughput"}[which]
        self.name = {"bake": "bake_uv_sphere_64x64_res128", "voxelize": "voxelize_torus_48x24_r2.5mm"}[which]

    def mesh(self):
        from pfsim import mesh as M

        return M.uv_sphere(0.5, 64, 64) if self.which == "bake" else M.torus(0.4, 0.12, 48, 24)

    def run_gpu(self, steps: int, warmup: int) -> dict:
        import torch

        from pfsim import mesh as M

        v, i = self.mesh()
        n_tri = len(i) // 3
        clocks = ClockSampler(torch.cuda.current_device())
        if self.which == "bake":
            run = lambda: M.bake_sdf(v, i, 128, None)
            points = 128 ** 3
        else:
            run = lambda: M.voxelize_mesh(v, i, 0.0025)
            ext = v.max(0).astype(np.float64) - v.min(0)
            points = int(np.prod(np.maximum(1, np.ceil(ext / 0.005))))
        for _ in range(warmup):
            run()
        torch.cuda.synchronize()
        clocks.start()
        t0 = time.perf_counter()
        for _ in range(steps):
            run()
        torch.cuda.synchronize()
        sec = (time.perf_counter() - t0) / steps
        return {"ms": sec * 1e3, "value": points * n_tri / sec, "points": points, "triangles": n_tri,
                "clocks": clocks.stop()}

    def run_cpu(self, threads: int, steps: int = 1) -> dict:
        """The oracle (one thread) on a bounded sample: the same mesh at a
        coarser grid (32^3 for the bake, 4x the particle radius for the
        voxeliser)."""
        from oracle import oracle as O

        v, i = self.mesh()
        n_tri = len(i) // 3
        t0 = time.perf_counter()
        if self.which == "bake":
            O.bake_sdf(v, i, 32, None)
            points = 32 ** 3
        else:
            O.voxelize_mesh(v, i, 0.01)
            ext = v.max(0).astype(np.float64) - v.min(0)
            points = int(np.prod(np.maximum(1, np.ceil(ext / 0.02))))
        sec = time.perf_counter() - t0
        return {"seconds_per_step": sec, "units_per_step": points * n_tri, "cores": 1,
                "sample": f"the same mesh on a coarser grid ({points} points), one pass, one thread"}


WORKLOADS = {"sort": SortWorkload, "batch": BatchWorkload, "serve": ServeWorkload, "dam": SceneWorkload,
             "mixed": SceneWorkload, "contacts": SceneWorkload, "cloth": SceneWorkload, "bake": MeshWorkload,
             "voxelize": MeshWorkload}


# -------------------------------------------------------------- ranks ----
def replica_seed(rank: int) -> int:
    """Seed of rank `rank`'s scene stream: replicas step disjoint scene sets
    (weak scaling, no data-path collective)."""
    return 1000 + rank


def max_over_ranks(values, device) -> list:
    """Element-wise maximum of per-rank timings (the job's time is its
    slowest rank's)."""
    import torch
    import torch.distributed as dist

    t = torch.tensor([float(v) for v in values], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return [float(v) for v in t.tolist()]


def sum_over_ranks(value, device) -> float:
    """The sum of a per-rank count (units every replica processed)."""
    import torch
    import torch.distributed as dist

    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.SUM)
    return float(t.item())


# -------------------------------------------------------------- main ----
def main() -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="pfsim", choices=["pfsim", "reference"])
    ap.add_argument("--workload", default="batch", choices=sorted(WORKLOADS))
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-plain", action="store_true", help="skip the plain per-scene baseline (profiling runs)")
    ap.add_argument("--scenes", type=int, default=256, help="scenes of the batch workload (smaller for profiling)")
    ap.add_argument("--live", type=int, default=96, help="steady-state live scenes of the serve workload")
    ap.add_argument("--no-serve", action="store_true", help="batch workload without its served arm")
    ap.add_argument("--serve-ticks", type=int, default=40, help="timed ticks of the batch workload's served arm")
    args = ap.parse_args()
    warmup = max(3, args.warmup)

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if args.workload == "batch":
        wl = WORKLOADS["batch"](args.scenes)
    elif args.workload == "serve":
        wl = WORKLOADS["serve"](args.live)
    elif args.workload in SceneWorkload.NAMES:
        wl = SceneWorkload(args.workload)
    elif args.workload in ("bake", "voxelize"):
        wl = MeshWorkload(args.workload)
    else:
        wl = WORKLOADS[args.workload]()

    if args.impl == "reference":
        if rank != 0:
            return
        threads = os.cpu_count() or 1
        cpu = wl.run_cpu(threads)
        value = cpu["units_per_step"] / cpu["seconds_per_step"]
        line = {
            "impl": "reference", "metric": wl.metric, "value": value, "unit": wl.unit, "n_gpus": args.gpus,
            "steps": args.steps, "warmup": warmup, "ms_per_step": cpu["seconds_per_step"] * 1e3,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "u32" if args.workload == "sort" else "f32", "data": "synthetic",
            "config": {"workload": wl.name},
            "cpu_baseline": {"value": value, "unit": wl.unit, "cores": cpu["cores"], "kind": "port", "sample": cpu["sample"]},
            "e2e": {"value": value, "unit": wl.unit, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        }
        print(json.dumps(line), flush=True)
        return

    import torch

    torch.cuda.set_device(local)
    if world > 1:
        import torch.distributed as dist
        from datetime import timedelta

        dist.init_process_group("nccl", timeout=timedelta(seconds=120), device_id=torch.device("cuda", local))

        def barrier():
            dist.barrier()
    else:

        def barrier():
            pass

    if args.workload in ("bake", "voxelize"):
        res = wl.run_gpu(args.steps, warmup)
        line = {"metric": wl.metric, "value": res["value"], "unit": wl.unit, "n_gpus": world, "steps": args.steps,
                "warmup": warmup, "ms_per_step": res["ms"], "higher_is_better": True, "scaling": "weak",
                "vs_baseline": None, "dtype": "f64", "data": "synthetic (procedural mesh)",
                "config": {"workload": wl.name, "points": res["points"], "triangles": res["triangles"]},
                "clocks": res["clocks"]}
        if rank == 0 and not args.no_cpu_baseline:
            cpu = wl.run_cpu(1)
            line["cpu_baseline"] = {"value": cpu["units_per_step"] / cpu["seconds_per_step"], "unit": wl.unit,
                                    "cores": cpu["cores"], "kind": "port", "sample": cpu["sample"]}
        if rank == 0:
            print(json.dumps(line), flush=True)
        return
    if args.workload in SceneWorkload.NAMES:
        res = wl.run_gpu(args.steps, warmup)
        line = {"metric": wl.metric, "value": res["value"], "unit": wl.unit, "n_gpus": world, "steps": args.steps,
                "warmup": warmup, "ms_per_step": res["ms"], "higher_is_better": True, "scaling": "weak",
                "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded)",
                "config": {"workload": wl.name, "particles": res["particles"]}, "clocks": res["clocks"]}
        if rank == 0 and not args.no_cpu_baseline:
            cpu = wl.run_cpu(os.cpu_count() or 1)
            line["cpu_baseline"] = {"value": cpu["units_per_step"] / cpu["seconds_per_step"], "unit": wl.unit,
                                    "cores": cpu["cores"], "kind": "port", "sample": cpu["sample"]}
        if rank == 0:
            print(json.dumps(line), flush=True)
        return
    if args.workload == "serve":
        res = wl.run_gpu(args.steps, warmup, rank, world, barrier, plain_baseline=not args.no_plain)
        line = {"metric": wl.metric, "value": res["units_per_step"] / (res["ms"] * 1e-3), "unit": wl.unit,
                "n_gpus": world, "steps": args.steps, "warmup": warmup, "ms_per_step": res["ms"],
                "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
                "data": "synthetic (seeded)", "config": {"workload": wl.name, "timing": "host wall clock per tick"},
                "clocks": res["clocks"]}
        line.update(res["extra"])
        if rank == 0:
            print(json.dumps(line), flush=True)
        return
    if args.workload == "batch":
        res = wl.run_gpu(args.steps, warmup, rank, world, barrier, plain_baseline=not args.no_plain)
    else:
        res = wl.run_gpu(args.steps, warmup, rank, world, barrier)
    ms = res["ms"]
    units = res["units_per_step"]  # this rank's; replicas step different scenes
    if world > 1:
        ms, e2e_ms = max_over_ranks([ms, res["e2e_ms"]], "cuda")
        units = sum_over_ranks(units, "cuda")
    else:
        e2e_ms = res["e2e_ms"]
    peak, peak_kind = hbm_peak()
    achieved = res["algorithmic_bytes"] / (res["kernel_ms"] * 1e-3) / 1e9
    value = units / (ms * 1e-3)
    line = {
        "metric": wl.metric, "value": value, "unit": wl.unit, "n_gpus": world, "steps": args.steps,
        "warmup": warmup, "ms_per_step": ms, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "u32", "data": "synthetic (seeded)",
        "config": {"workload": wl.name, "inputs_larger_than_l2": True, "parallelism": f"replicas x{world}"},
        "roofline": {"bound": "hbm", "kernel": res["kernel_name"], "achieved": achieved, "peak": peak,
                     "peak_kind": peak_kind, "unit": "GB/s", "frac": achieved / peak,
                     "traffic": res.get("traffic")},
        "e2e": {"value": units / (e2e_ms * 1e-3), "unit": wl.unit,
                "h2d_bytes_per_step": res["h2d"], "d2h_bytes_per_step": res["d2h"]},
        "gpu_launches": res["gpu_launches_per_step"] * args.steps,
        "clocks": res["clocks"],
    }
    line["dtype"] = "u32" if args.workload == "sort" else "f32"
    if "stages" in res:
        line["roofline"]["stages"] = res["stages"]
    line.update(res.get("extra", {}))
    if args.workload == "batch" and not args.no_serve and world == 1:
        # the served half of the metric: the Poisson request stream, batched
        # (cohorts, graphs) against the plain per-scene loop, on this GPU
        sv = WORKLOADS["serve"](args.live)
        sres = sv.run_gpu(args.serve_ticks, 5, rank, world, barrier, plain_baseline=not args.no_plain)
        ex = sres["extra"]
        line["served"] = {
            "workload": sv.name, "ticks": args.serve_ticks, "value": sres["units_per_step"] / (sres["ms"] * 1e-3),
            "unit": wl.unit, "p50_tick_ms": ex["p50_tick_ms"], "p99_tick_ms": ex["p99_tick_ms"],
            "plain_value": ex["plain_value"], "plain_p50_tick_ms": ex["plain_p50_tick_ms"],
            "plain_p99_tick_ms": ex["plain_p99_tick_ms"], "served_over_plain": ex["served_over_plain"],
            "plain_with_builds_value": ex["plain_with_builds_value"],
            "plain_with_builds_p99_tick_ms": ex["plain_with_builds_p99_tick_ms"],
            "timing": "host wall clock per tick; the plain arm's ticks without its world builds",
            "cohort_builds": ex["cohort_builds"], "max_swap_ms": ex["max_swap_ms"],
            "max_step_ms": ex["max_step_ms"], "max_free_ms": ex["max_free_ms"],
            "clocks": sres["clocks"],
        }
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        cpu = wl.run_cpu(os.cpu_count() or 1)
        line["cpu_baseline"] = {"value": cpu["units_per_step"] / cpu["seconds_per_step"], "unit": wl.unit,
                                "cores": cpu["cores"], "kind": "port", "sample": cpu["sample"]}
    if rank == 0:
        print(json.dumps(line), flush=True)
    if world > 1:
        import torch.distributed as dist

        dist.destroy_process_group()


if __name__ == "__main__":
    main()
