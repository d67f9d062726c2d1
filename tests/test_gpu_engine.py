"""GPU: the batch engine (persistent kernels over many cases, CUDA-graph
launches, continuous admission).  A case's result must not depend on which
other cases share the GPU (bit for bit), and must equal the same case run
alone through the one-case operator (thx_rk3_steps): bit for bit in FP64,
within FP32 round-off in FP32-mixed, where the batched and one-case kernels
are separate compilations free to contract multiply-adds differently."""
import numpy as np
import pytest

import theseus_b200 as T
from theseus_b200 import cases
from theseus_b200.serving import BatchEngine, Case, SyntheticStream, serve
from _helpers import to_dev

pytestmark = pytest.mark.gpu

FLUX = dict(numerical_flux="chandrashekar", surface_flux="roe")


def vortex_case(dim, order, n, viscous, nsteps, mach=0.5, strength=3.0, seed=0):
    lo, hi = [-5.0] * dim, [5.0] * dim
    m = T.periodic_box(dim, order, n, lo, hi)
    c = np.sqrt(1.4)
    v = mach * c / np.sqrt(2.0)
    u0 = cases.isentropic_vortex(m.coords, strength=strength, u_inf=(v, v))
    if dim == 3:
        u0 = u0  # isentropic_vortex adds w = 0 in 3-D
    rng = np.random.default_rng(seed)
    u0 = u0 * (1.0 + 1e-3 * rng.uniform(-1, 1, u0.shape))
    E = 1.0 / 0.4 + v * v
    off = (1.0, v, v, E, 0.0) if dim == 2 else (1.0, v, v, 0.0, E)
    h = 10.0 / n[0]
    dt = 0.4 * h / ((2 * order + 1) * (np.sqrt(2) * v + c + 1.0))
    return Case(mesh=m, u0=u0, nsteps=nsteps, dt=dt, viscous=viscous, mu=0.01 if viscous else 0.0,
                Pr=0.72, state_offset=off)


def field_errors(a, b, dim):
    """Relative L2 error per conserved field (density, momentum vector, energy)."""
    a = a.reshape(a.shape[0], -1)
    b = b.reshape(b.shape[0], -1)
    groups = [[0], list(range(1, dim + 1)), [dim + 1]]
    return np.array([np.sqrt(((a[g] - b[g]) ** 2).sum() / (b[g] ** 2).sum()) for g in groups])


def alone(case, precision):
    import torch
    cls = T.NSOperator if case.viscous else T.EulerOperator
    kw = dict(FLUX, precision=precision, mu=case.mu, Pr=case.Pr)
    if precision == "fp32":
        kw["state_offset"] = list(case.state_offset)
    op = cls(case.mesh, **kw)
    u = to_dev(case.u0, torch.float64)
    op.rk3_steps(u, case.dt, case.nsteps)
    torch.cuda.synchronize()
    return u.cpu().numpy()


def run_engine(engine, batch):
    ids = {engine.admit(c): i for i, c in enumerate(batch)}
    assert None not in ids
    out = [None] * len(batch)
    for _ in range(100000):
        if not ids:
            break
        engine.advance()
        for cid in engine.poll():
            i = ids.pop(cid)
            out[i] = engine.fetch(cid, batch[i].u0.shape)
    assert not ids
    return out


@pytest.mark.parametrize("precision", ["fp32", "fp64"])
def test_engine_shared_geometry(cuda, precision):
    """Cases that name the same mesh with a geometry key share one device copy
    of its geometry; their results equal those of cases with their own copies,
    bit for bit, and a key reused with a different mesh size is refused."""
    import dataclasses
    base = [vortex_case(2, 3, (6, 6), v, 15, seed=i) for i, v in enumerate((False, True, False))]
    mesh = base[0].mesh
    base = [dataclasses.replace(c, mesh=mesh) for c in base]
    keyed = [dataclasses.replace(c, geometry_key=7) for c in base]
    eng = BatchEngine(precision=precision, steps_per_launch=5, **FLUX)
    try:
        own = run_engine(eng, base)
        shared = run_engine(eng, keyed)
    finally:
        eng.close()
    for a, b in zip(own, shared):
        assert np.array_equal(a, b)
    eng = BatchEngine(precision=precision, steps_per_launch=5, **FLUX)
    try:
        run_engine(eng, keyed[:1])
        other = dataclasses.replace(vortex_case(2, 3, (5, 6), False, 5), geometry_key=7)
        with pytest.raises(T.THXError):
            eng.admit(other)
    finally:
        eng.close()


MIX = [(2, 2, (6, 6), False, 20), (2, 3, (5, 7), True, 20), (2, 5, (4, 4), False, 25),
       (2, 2, (8, 5), False, 30), (3, 3, (2, 2, 3), True, 10), (2, 4, (3, 3), True, 7)]


@pytest.mark.parametrize("precision", ["fp32", "fp64"])
def test_engine_matches_one_case_runs(cuda, precision):
    batch = [vortex_case(*spec, seed=i) for i, spec in enumerate(MIX)]
    eng = BatchEngine(precision=precision, steps_per_launch=10, **FLUX)
    got = run_engine(eng, batch)
    for c, g in zip(batch, got):
        ref = alone(c, precision)
        if precision == "fp64":
            assert np.array_equal(g, ref), np.abs(g - ref).max()
        else:
            err = field_errors(g, ref, c.mesh.dim)
            assert err.max() <= 1e-5, err
    st = eng.stats()
    assert st["active_cases"] == 0 and st["cases_done"] == len(batch) and st["bytes_in_use"] == 0
    eng.close()


def test_engine_grid_tuning(cuda):
    """The online tuner searches the elements per CTA and the volume, face and
    (Navier-Stokes) gradient grids of each batch group; the result stays
    bit-identical to the one-case run whatever configuration the launches
    used."""
    import torch
    sms = torch.cuda.get_device_properties(0).multi_processor_count
    batch = [vortex_case(2, 3, (6, 6), True, 300, seed=1), vortex_case(2, 3, (5, 7), True, 300, seed=2),
             vortex_case(2, 4, (6, 6), False, 300, seed=3)]
    eng = BatchEngine(precision="fp64", steps_per_launch=3, **FLUX)
    ids = {eng.admit(c): i for i, c in enumerate(batch)}
    seen = None
    out = [None] * len(batch)
    for _ in range(100000):
        if not ids:
            break
        eng.advance()
        if len(ids) == len(batch):
            seen = eng.groups()
        for cid in eng.poll():
            i = ids.pop(cid)
            out[i] = eng.fetch(cid, batch[i].u0.shape)
    assert seen is not None and len(seen) == 2
    ns = {g["navier_stokes"]: g for g in seen}
    assert set(ns) == {0, 1}
    for g in seen:
        assert g["dim"] == 2 and g["order"] in (3, 4)
        assert g["volume_grid"] in (sms, 2 * sms, 4 * sms)
        assert g["face_grid"] in (4 * sms, 8 * sms, 16 * sms)
        full = max(1, 256 // (g["order"] + 1) ** g["dim"])
        assert g["elements_per_block"] in (full, full // 2)
    assert ns[1]["gradient_grid"] in (sms, 2 * sms, 4 * sms) and ns[0]["gradient_grid"] == 0
    final = eng.groups()
    # 100 launches per group are far more than the 22 timed ones the search needs
    assert all(g["tuned"] == 1 and g["active_cases"] == 0 and g["best_cost_ms"] > 0 for g in final), final
    for c, g in zip(batch, out):
        assert np.array_equal(g, alone(c, "fp64"))
    eng.close()


def test_engine_result_independent_of_the_mix(cuda):
    target = vortex_case(2, 3, (5, 5), True, 20, seed=42)
    e1 = BatchEngine(precision="fp32", steps_per_launch=5, **FLUX)
    only = run_engine(e1, [target])[0]
    e1.close()
    others = [vortex_case(*spec, seed=10 + i) for i, spec in enumerate(MIX)]
    e2 = BatchEngine(precision="fp32", steps_per_launch=5, **FLUX)
    mixed = run_engine(e2, others[:3] + [target] + others[3:])[3]
    e2.close()
    assert np.array_equal(only, mixed)


def test_engine_budget_admission(cuda):
    a = vortex_case(2, 3, (6, 6), False, 10)
    b = vortex_case(2, 3, (6, 6), False, 10, seed=1)
    eng = BatchEngine(precision="fp32", steps_per_launch=10, hbm_budget=1, **FLUX)
    assert eng.admit(a) is None                      # nothing fits a 1-byte budget
    eng.close()
    probe = BatchEngine(precision="fp32", steps_per_launch=10, **FLUX)
    need = probe.footprint(a)
    probe.close()
    eng = BatchEngine(precision="fp32", steps_per_launch=10, hbm_budget=need + need // 2, **FLUX)
    ida = eng.admit(a)
    assert ida is not None and eng.admit(b) is None  # one fits, two do not
    out = run_engine_ids(eng, {ida: a})
    assert eng.admit(b) is not None                  # room again after the fetch
    assert field_errors(out[ida], alone(a, "fp32"), 2).max() <= 1e-5
    eng.close()


def run_engine_ids(engine, idmap):
    out = {}
    while len(out) < len(idmap):
        engine.advance()
        for cid in engine.poll():
            out[cid] = engine.fetch(cid, idmap[cid].u0.shape)
    return out


def test_serving_loop_small_stream(cuda):
    stream = SyntheticStream(8, rate=4000.0, seed=3, sides=(4, 10), orders=(2, 5), nsteps=20)
    reqs = [stream.case(i) for i in range(8)]
    eng = BatchEngine(precision="fp32", steps_per_launch=10, **FLUX)
    results, lat, makespan = serve(eng, reqs)
    eng.close()
    assert all(r is not None for r in results)
    assert np.all(lat > 0) and makespan > 0
    for r, c in zip(results, reqs):
        assert field_errors(r, alone(c, "fp32"), 2).max() <= 1e-5
        assert field_errors(r, alone(c, "fp64"), 2).max() <= 1e-5
        assert np.all(np.isfinite(r))
