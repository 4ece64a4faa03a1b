"""Continuous batching: stepwise batch runs (fv_batch_begin / _advance /
_report) and waves rebuilt mid-flight with the running problems carried over.

- a problem admitted into a running wave, and the problems it joins, give the
  same bits (solution and iteration count) as each alone in fv_batch_cg /
  fv_batch_bicgstab: CG + IC(0) and BiCGStab + ILU(0), FP64 and mixed
  precision, box-colour ordering per problem
- the same through the server's WaveRun over generated requests
- invalid carries are refused
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _square(fv, side, seed):
    m = fv.Mesh.square(side, 0.2, seed)
    kf, _, sc = m.fields(seed, 1.0, 0.5 + (seed % 7) * 0.2, source_const=1.0)
    return m, kf, None, sc


def _cube(fv, n, seed):
    m = fv.Mesh.cube(n, 0.15, seed)
    kappa0 = float(np.linalg.norm((1.0, 0.5, 0.25))) / n / 3.0
    kf, fl, sc = m.fields(seed, kappa0, 0.5, velocity=(1.0, 0.5, 0.25), source_uniform=True)
    return m, kf, fl, sc


def _system(fv, probs, ordering):
    from fvb200.batch import MeshBatch
    mb = MeshBatch([p[0] for p in probs])
    kf = mb.face_field([p[1] for p in probs])
    sc = mb.cell_field([p[3] for p in probs])
    nb = mb.n_boundary_faces
    if probs[0][2] is None:
        eq = -fv.laplacian(fv.Orthogonal(), kf) - fv.source(sc)
        make = fv.IncompleteCholesky
    else:
        fl = mb.face_field([p[2] for p in probs])
        eq = fv.convection(fv.Upwind(fl), fl) - fv.laplacian(fv.Orthogonal(), kf) - fv.source(sc)
        make = fv.IncompleteLowerUpper
    A, b = fv.assemble(eq, (np.zeros(nb), np.zeros(nb)), mb)
    P = make.from_matrix(A, 0, ordering=ordering, offsets=mb.cell_offsets if ordering else None)
    x = fv.DistributedVector.from_size(mb.n_cells)
    return dict(mb=mb, A=A, b=b, P=P, x=x)


OPTS = dict(relative_tolerance=1e-9, absolute_tolerance=1e-9, outer_tolerance=1e-10, inner_relative_tolerance=1e-2,
            max_iterations=4000)


def _alone(fv, prob, solver, precision, ordering, tile):
    from fvb200.batch import BatchCG
    s = _system(fv, [prob], ordering)
    out = BatchCG(s["A"], s["mb"].cell_offsets, tile).solve(s["P"], s["b"], s["x"], precision=precision,
                                                            solver=solver, **OPTS)
    assert out["fp64_fallback"][0] == 0
    return s["x"].numpy().copy(), int(out["iterations"][0])


@pytest.mark.parametrize("solver,precision", [("cg", "fp64"), ("cg", "mixed"), ("bicgstab", "fp64"),
                                              ("bicgstab", "mixed")])
def test_admitted_mid_flight_same_as_alone(fv, solver, precision):
    """Wave 1 = {a, b, c} runs some iterations; wave 2 = {d, c, a} (b finished
    or dropped, d admitted) carries a and c over at new positions; after more
    iterations wave 3 = {e, c} carries c over again.  Every problem's solution
    and iteration count are the bits of its solve alone."""
    from fvb200.batch import BatchCG
    ordering, tile = "boxes", 256
    if solver == "cg":
        probs = {k: _square(fv, s, 40 + i) for i, (k, s) in enumerate(zip("abcde", [14, 9, 20, 11, 16]))}
    else:
        probs = {k: _cube(fv, n, 60 + i) for i, (k, n) in enumerate(zip("abcde", [8, 5, 16, 6, 10]))}
    alone = {k: _alone(fv, p, solver, precision, ordering, tile) for k, p in probs.items()}
    group = 8 if solver == "cg" else 4  # iterations per advance group
    # c runs in three waves: 8 iterations, one group, then the rest
    assert alone["c"][1] > 8 + 2 * group
    kw = dict(precision=precision, solver=solver, **{k: v for k, v in OPTS.items()})
    got = {}

    def collect(wave, names, bc, only=None):
        running, done = bc.advance(0)
        rep = bc.report()
        xs = wave["x"].numpy()
        off = wave["mb"].cell_offsets
        for k, name in enumerate(names):
            if done[k] and name not in got and (only is None or name in only):
                assert rep["fp64_fallback"][k] == 0 and rep["status"][k] == 0
                got[name] = (xs[off[k]:off[k + 1]].copy(), int(rep["iterations"][k]))
        return done

    names1 = ["a", "b", "c"]
    w1 = _system(fv, [probs[k] for k in names1], ordering)
    b1 = BatchCG(w1["A"], w1["mb"].cell_offsets, tile)
    b1.begin(w1["P"], w1["b"], w1["x"], **kw)
    running, done = b1.advance(8)
    assert running == 3 and not done.any()
    collect(w1, names1, b1)

    names2 = ["d", "c", "a"]
    w2 = _system(fv, [probs[k] for k in names2], ordering)
    b2 = BatchCG(w2["A"], w2["mb"].cell_offsets, tile)
    b2.begin(w2["P"], w2["b"], w2["x"], carry_from=b1, carry=[-1, 2, 0], **kw)
    b1.close()
    rep = b2.report()
    assert rep["iterations"][1] >= 8 and rep["iterations"][2] >= 8 and rep["iterations"][0] == 0
    b2.advance(group)
    done2 = collect(w2, names2, b2)
    assert not done2[1], "c must still be running to be carried again"

    names3 = ["e", "c"]
    w3 = _system(fv, [probs[k] for k in names3], ordering)
    b3 = BatchCG(w3["A"], w3["mb"].cell_offsets, tile)
    b3.begin(w3["P"], w3["b"], w3["x"], carry_from=b2, carry=[-1, 1], **kw)
    # d and a finish in wave 2; c's result is taken from wave 3 only
    for _ in range(1000):
        collect(w2, names2, b2, only=("d", "a"))
        if "d" in got and "a" in got:
            break
        b2.advance(64)
    for _ in range(1000):
        if b3.advance(64)[0] == 0:
            break
    collect(w3, names3, b3)
    b2.close()
    b3.close()
    assert set(got) == {"a", "c", "d", "e"}  # b never finished: it was left behind in wave 1
    for name, (x, its) in got.items():
        xa, ia = alone[name]
        assert its == ia, name
        assert np.array_equal(x, xa), name


def test_wave_run_refill_same_as_alone(fv):
    """The server's WaveRun: requests admitted into a running wave give the
    bits of their wave alone (FP64 and mixed)."""
    from fvb200.serve import MeshCache, Request, WaveRun, solve_wave
    import torch
    cache = MeshCache(fv)
    st = torch.cuda.Stream()
    for precision in ("fp64", "mixed"):
        reqs = [Request(k, 0.0, "2d", side, 1000 + k, cells=2 * side * side)
                for k, side in enumerate([24, 40, 16, 32])]
        alone = {}
        for r in reqs:
            q = Request(r.rid, 0.0, r.kind, r.side, r.seed, cells=r.cells)
            solve_wave(fv, cache, [q], st, keep_solution=True, precision=precision)
            alone[r.rid] = (q.solution, q.iterations)
        run = WaveRun(fv, cache, reqs[:2], st, precision=precision, keep_solution=True)
        finished = []
        for _ in range(2):
            f, s = run.advance(8)
            assert not s
            finished += f
        nxt = WaveRun(fv, cache, run.running() + reqs[2:], st, prev=run, precision=precision, keep_solution=True)
        run.close()
        while nxt.running():
            f, s = nxt.advance(32)
            assert not s
            finished += f
        nxt.close()
        assert sorted(r.rid for r in finished) == [0, 1, 2, 3]
        for r in finished:
            xa, ia = alone[r.rid]
            assert r.iterations == ia and np.array_equal(r.solution, xa), (precision, r.rid)
            assert r.fields is None


def test_invalid_carry_is_refused(fv):
    from fvb200._lib import FV_ERR_INVALID, FvError
    from fvb200.batch import BatchCG
    p1, p2 = _square(fv, 10, 5), _square(fv, 12, 6)
    w1 = _system(fv, [p1, p2], None)
    b1 = BatchCG(w1["A"], w1["mb"].cell_offsets, 256)
    b1.begin(w1["P"], w1["b"], w1["x"], precision="fp64", **{k: OPTS[k] for k in ("relative_tolerance",
                                                                                 "absolute_tolerance")})
    b1.advance(8)
    w2 = _system(fv, [p2, p1], None)
    cases = [
        (BatchCG(w2["A"], w2["mb"].cell_offsets, 256), [0, 1], "fp64"),    # sizes swapped
        (BatchCG(w2["A"], w2["mb"].cell_offsets, 512), [1, 0], "fp64"),    # another tile partition
        (BatchCG(w2["A"], w2["mb"].cell_offsets, 256), [1, 1], "fp64"),    # the same problem twice
        (BatchCG(w2["A"], w2["mb"].cell_offsets, 256), [1, 0], "mixed"),   # another precision
    ]
    for bc, carry, precision in cases:
        with pytest.raises(FvError) as e:
            bc.begin(w2["P"], w2["b"], w2["x"], precision=precision, carry_from=b1, carry=carry)
        assert e.value.status == FV_ERR_INVALID
    ok = BatchCG(w2["A"], w2["mb"].cell_offsets, 256)
    ok.begin(w2["P"], w2["b"], w2["x"], precision="fp64", carry_from=b1, carry=[1, 0],
             relative_tolerance=OPTS["relative_tolerance"], absolute_tolerance=OPTS["absolute_tolerance"])
    while ok.advance(64)[0]:
        pass
    # a finished problem cannot be carried
    ok2 = BatchCG(w2["A"], w2["mb"].cell_offsets, 256)
    with pytest.raises(FvError):
        ok2.begin(w2["P"], w2["b"], w2["x"], precision="fp64", carry_from=ok, carry=[0, -1])


def test_merged_mesh_orders_equal_the_union_order(fv):
    """A wave's order merged from its meshes' own orders (each computed once
    per mesh) is the order fv_order_boxes gives the union, 2D and 3D."""
    from fvb200.serve import mesh_order
    for probs in ([_square(fv, s, 80 + s) for s in (12, 30, 7, 21)], [_cube(fv, n, 90 + n) for n in (5, 9, 3)]):
        w = _system(fv, probs, None)
        ref, info = fv.order_boxes(w["A"], offsets=w["mb"].cell_offsets)
        merged = fv.merge_orders([mesh_order(fv, p[0]) for p in probs], w["mb"].cell_offsets)
        assert np.array_equal(merged, ref)
        # the levels reported for one mesh alone are those of its reordered factor
        perm, _, lev = fv.order_boxes(_system(fv, probs[1:2], None)["A"], levels=True)
        assert np.all(np.diff(lev) >= 0) and lev[0] == 0
        P = (fv.IncompleteCholesky if probs[0][2] is None else fv.IncompleteLowerUpper).from_matrix(
            _system(fv, probs[1:2], None)["A"], 0, ordering=perm)
        assert P.levels()[2] == int(lev[-1]) + 1
