"""Batched ensembles, the continuous-batching server and the launch-shape autotuner.

The property every multi-solve path must keep: each solve's result is bitwise the result
of the same solve stepped alone (no shared state, fixed-order reductions), whatever else
runs beside it -- checked with np.array_equal, not a tolerance.
"""
import math

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

FP64, FP32 = 0, 1


@pytest.fixture(scope="module")
def mod():
    import spectral_solver_b200 as m
    return m


def ensemble_specs(count, seed=2026):
    """Uneven sizes and Reynolds numbers, seeded perturbations, CFL-limited steps (the
    ensemble configuration's recipe at a smaller count)."""
    rng = np.random.default_rng(seed)
    specs = []
    for i in range(count):
        n = int(rng.choice([32, 48, 64, 96, 128]))
        re = float(np.exp(rng.uniform(np.log(400.0), np.log(3200.0))))
        specs.append(dict(n=n, nu=1.0 / re, precision=FP64 if i % 2 == 0 else FP32, seed=i, pert_amp=1e-3,
                          pert_kmax=max(1, n // 8), dt=0.0, cfl=0.5, dt_max=0.5))
    return specs


def test_batch_matches_solves_alone(mod):
    specs = ensemble_specs(8)
    with mod.Batch(specs) as b:
        b.step(3)
        got = [b.solver(i).get_state() for i in range(len(specs))]
        dts = b.dt
    for i, sp in enumerate(specs):
        with mod.Solver(sp["n"], 1.0 / sp["nu"], seed=sp["seed"], pert_amp=sp["pert_amp"], pert_kmax=sp["pert_kmax"],
                        precision=sp["precision"]) as s:
            # every member takes the CFL step from its current vmax at every step
            host_cfl_loop(s, sp["n"], float("inf"), 3, sp["cfl"], sp["dt_max"])
            assert s.host_dts[0] == dts[i]
            ref = s.get_state()
        for a, r in zip(got[i], ref):
            assert np.array_equal(a, r), (i, sp["n"], sp["precision"])


def test_batch_timing_and_fixed_dt(mod):
    specs = [dict(n=64, nu=1 / 1600.0, dt=5e-3), dict(n=48, nu=1 / 800.0, dt=2e-3, precision=FP32)]
    with mod.Batch(specs) as b:
        assert b.dt == [5e-3, 2e-3]
        ms = b.time_steps(4)
        assert ms > 0.0
        d = b.solver(0).diagnostics(0.02)
    with mod.Solver(64, 1600.0) as s:
        s.step(5e-3, 4)
        assert s.diagnostics(0.02)["kinetic_energy"] == d["kinetic_energy"]


def host_cfl_loop(s, n, t_end, max_steps, cfl=0.5, dt_max=0.5):
    """The reference's adaptive loop (run_taylor_green, ava_taylor_green_impl.hpp:1363-1378)
    on the host: vmax of the current state, dt = min(dt_max, cfl dx / vmax) clipped to the
    horizon, one step.  Returns (steps, t) and the step sizes in s.host_dts."""
    dx = 2.0 * math.pi / n
    t, steps, dts = 0.0, 0, []
    while t < t_end - 1e-14 and steps < max_steps:
        vmax = s.max_velocity()
        main_dt = dt_max
        if vmax > 1e-14:
            main_dt = min(main_dt, cfl * dx / vmax)
        dt = min(main_dt, t_end - t)
        s.step(dt)
        t += dt
        steps += 1
        dts.append(dt)
    s.host_dts = dts
    return steps, t


def run_server(mod, requests, budget, precision=FP32):
    done = {}
    max_resident = 0
    with mod.Server(budget, precision) as srv:
        ids = [srv.submit(**r) for r in requests]
        for _ in range(100000):
            out, res, q, used = srv.step()
            max_resident = max(max_resident, res)
            assert used <= budget
            for r in out:
                done[r["id"]] = r
            if len(done) == len(requests):
                break
    return [done[i] for i in ids], max_resident


def test_server_result_same_alone_and_in_mix(mod):
    # a small solve takes up to 64 steps per tick (N_max^3 / N^3), so the horizons are long
    # enough that the requests stay resident together for several ticks
    a = dict(n=64, nu=1 / 1000.0, t_end=2.0, seed=7, pert_amp=1e-3, pert_kmax=8)
    others = [dict(n=32, nu=1 / 500.0, t_end=9.0, seed=1, pert_amp=1e-3, pert_kmax=4),
              dict(n=128, nu=1 / 2000.0, t_end=0.6, seed=2, pert_amp=1e-3, pert_kmax=16),
              dict(n=48, nu=1 / 700.0, t_end=3.0, seed=3, pert_amp=1e-3, pert_kmax=6)]
    budget = 8 << 30
    alone, _ = run_server(mod, [a], budget)
    mixed, max_res = run_server(mod, others[:1] + [a] + others[1:], budget)
    assert max_res >= 2  # the requests really overlapped on the device
    assert mixed[1]["steps"] == alone[0]["steps"] and mixed[1]["dt"] == alone[0]["dt"]
    for key in ("kinetic_energy", "dissipation", "enstrophy", "max_velocity"):
        assert mixed[1]["final"][key] == alone[0]["final"][key], key
    # and the same as a handle stepped by the reference's adaptive loop on the host
    with mod.Solver(64, 1000.0, seed=7, pert_amp=1e-3, pert_kmax=8, precision=FP32) as s:
        steps, t = host_cfl_loop(s, 64, a["t_end"], 10 ** 9)
        assert steps == alone[0]["steps"]
        assert s.diagnostics(a["t_end"])["kinetic_energy"] == alone[0]["final"]["kinetic_energy"]


def test_server_admits_by_budget(mod):
    per = mod.load().sns_bytes_required(64, FP32)
    reqs = [dict(n=64, nu=1 / 1600.0, t_end=0.05, seed=i) for i in range(3)]
    res, max_res = run_server(mod, reqs, budget=int(per * 1.5))
    assert max_res == 1 and len(res) == 3
    assert all(r["final"]["kinetic_energy"] > 0 for r in res)


@pytest.mark.parametrize("n,precision", [(64, FP64), (256, FP32)])
def test_autotune_cache_and_parity(mod, tmp_path, n, precision):
    from oracle.ref_r2c import TaylorGreenR2C, half_to_full
    cache = str(tmp_path / "autotune.txt")
    with mod.Solver(n, 1600.0, precision=precision) as s:
        cfg = s.autotune(2, cache)
    with open(cache) as f:
        assert len(f.read().splitlines()) == 1
    with mod.Solver(n, 1600.0, precision=precision) as s2:
        assert s2.autotune(2, cache) == cfg  # read from the cache
        o = TaylorGreenR2C(n, 1600.0)
        r_ref = [half_to_full(c) for c in o.compute_rhs()]
        r = s2.rhs([half_to_full(c) for c in o.u_hat])
    num = sum(float(np.sum(np.abs(x - y) ** 2)) for x, y in zip(r, r_ref))
    den = sum(float(np.sum(np.abs(y) ** 2)) for y in r_ref)
    assert math.sqrt(num / den) < (1e-12 if precision == FP64 else 2e-5)


def test_server_reuses_retired_handles(mod):
    """Retired solves leave their device memory in an idle pool and later requests of the
    same N take it over: five 32^3 requests under a budget of two handles allocate two, and
    each result is bitwise that of the request served alone by a fresh server."""
    per = mod.load().sns_bytes_required(32, FP32)
    reqs = [dict(n=32, nu=1 / (400.0 + 100 * i), t_end=0.3 + 0.1 * i, seed=20 + i, pert_amp=1e-3, pert_kmax=4)
            for i in range(5)]
    budget = int(per * 2.5)
    done = {}
    with mod.Server(budget, FP32) as srv:
        ids = [srv.submit(**r) for r in reqs]
        for _ in range(200000):
            out, res, q, used = srv.step()
            assert used <= budget
            for r in out:
                done[r["id"]] = r
            if len(done) == len(reqs):
                break
        stats = srv.stats()
    assert stats["handles_created"] == 2
    assert stats["idle_bytes"] == 2 * per
    for i, r in zip(ids, reqs):
        alone, _ = run_server(mod, [r], budget)
        assert done[i]["steps"] == alone[0]["steps"]
        for key in ("kinetic_energy", "dissipation", "enstrophy", "max_velocity"):
            assert done[i]["final"][key] == alone[0]["final"][key], key


def test_server_mixed_sizes_wait_for_their_handles(mod):
    """Alternating 32^3 and 48^3 requests under a budget of one handle of each: a request
    whose N has a resident solve waits for that handle instead of freeing the idle handle of
    the other size and allocating (cudaFree / cudaMalloc synchronise the device), so eight
    requests are served by the two handles created at the start."""
    lib = mod.load()
    per32, per48 = lib.sns_bytes_required(32, FP32), lib.sns_bytes_required(48, FP32)
    reqs = []
    for i in range(8):
        n = 32 if i % 2 == 0 else 48
        reqs.append(dict(n=n, nu=1 / (400.0 + 50 * i), t_end=0.2 + 0.15 * ((i * 5) % 4), seed=40 + i,
                         pert_amp=1e-3, pert_kmax=4))
    budget = per32 + per48
    done = {}
    with mod.Server(budget, FP32) as srv:
        ids = [srv.submit(**r) for r in reqs]
        for _ in range(400000):
            out, res, q, used = srv.step()
            assert used <= budget
            for r in out:
                done[r["id"]] = r
            if len(done) == len(reqs):
                break
        stats = srv.stats()
    assert len(done) == len(reqs)
    assert stats["handles_created"] == 2
    assert all(np.isfinite(done[i]["final"]["kinetic_energy"]) for i in ids)


@pytest.mark.parametrize("precision", [FP64, FP32])
def test_device_clock_matches_host_adaptive_loop(mod, precision):
    """sns_step_cfl takes the reference's adaptive step on the device: the same step sizes,
    time and state, bit for bit, as the host loop over sns_max_velocity and sns_step; it
    stops exactly at the horizon and later steps leave the state as it is."""
    n, t_end = 48, 0.6
    with mod.Solver(n, 900.0, seed=4, pert_amp=1e-2, pert_kmax=5, precision=precision) as host:
        steps, t = host_cfl_loop(host, n, t_end, 10 ** 6)
        ref = host.get_state()
        dts = host.host_dts
    with mod.Solver(n, 900.0, seed=4, pert_amp=1e-2, pert_kmax=5, precision=precision) as dev:
        dev.set_clock(0.0, t_end, 0.5, 0.5)
        for k in range(steps):
            dev.step_cfl(1)
            c = dev.clock()
            assert c["dt"] == dts[k] and not c["stopped"], k
        c = dev.clock()
        assert c["t"] == t and c["steps"] == steps
        dev.step_cfl(3)  # past the horizon: no-ops
        c = dev.clock()
        assert c["stopped"] and c["steps"] == steps
        got = dev.get_state()
    assert all(np.array_equal(a, b) for a, b in zip(got, ref))


def test_batch_cfl_member_steps_like_host_loop(mod):
    """A batch member with dt <= 0 takes the CFL step from its own vmax at every step, on
    the device, inside the batch graph: after 15 batch steps its clock and state equal the
    host adaptive loop's (no horizon)."""
    specs = [dict(n=48, nu=1 / 700.0, dt=0.0, cfl=0.5, dt_max=0.5, seed=3, pert_amp=1e-2, pert_kmax=5),
             dict(n=32, nu=1 / 500.0, dt=4e-3, seed=1, pert_amp=1e-3, pert_kmax=4)]
    with mod.Batch(specs) as b:
        b.step(15)
        c = b.solver(0).clock()
        got = b.solver(0).get_state()
        first_dt = b.dt[0]
    with mod.Solver(48, 700.0, seed=3, pert_amp=1e-2, pert_kmax=5) as s:
        steps, t = host_cfl_loop(s, 48, float("inf"), 15)
        ref = s.get_state()
        assert s.host_dts[0] == first_dt
    assert c["steps"] == 15 and c["t"] == t
    assert all(np.array_equal(a, b) for a, b in zip(got, ref))
