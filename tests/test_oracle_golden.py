"""The CPU oracle (C restatement) pinned against the reference.

Golden fixtures in tests/golden/ were produced by running the reference's own
sources (tests/golden/gen_golden.py). The restatement must reproduce every
stored intermediate and final array to 1e-13 relative L2 (in practice ~1e-15:
the two differ only in summation order), and the reference library itself is
re-run where it was built.
"""
import glob
import os

import numpy as np
import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
GOLDEN = sorted(glob.glob(os.path.join(HERE, "golden", "ref*.npz")))
TOL = 1e-13


def rel(a, b):
    nb = np.linalg.norm(b)
    return np.linalg.norm(np.asarray(a) - np.asarray(b)) / (nb if nb > 0 else 1.0)


def load_case(path):
    from oracle import PANEL2_DTYPE, PANEL3_DTYPE, PAIR_DTYPE
    z = np.load(path)
    dim, n, seed, deg, leaf, ns = (int(v) for v in z["params"])
    theta, eps = (float(v) for v in z["fparams"])
    pdt = PANEL2_DTYPE if dim == 2 else PANEL3_DTYPE
    tg = tuple(z[f"t{d}"] for d in range(dim))
    split = ns > 0
    sc = tuple(z[f"s{d}"] for d in range(dim)) if split else tg
    S = "S" if split else "T"
    tree = {"dim": dim, "degree": deg, "eps": eps, "thresh": leaf, "targets": tg, "sources": sc,
            "panels_t": z["T_panels"].view(pdt), "panels_s": z[f"{S}_panels"].view(pdt),
            "level_start_t": z["T_level_start"], "level_start_s": z[f"{S}_level_start"],
            "leaf_of_s": z[f"{S}_leaf_of"], "inside_t": z["T_inside"], "inside_s": z[f"{S}_inside"]}
    for k in ("pp", "pc", "cp", "cc"):
        tree[k] = z[k].view(PAIR_DTYPE)
    return z, tree, dict(dim=dim, n=n, deg=deg, leaf=leaf, theta=theta, eps=eps, split=split)


@pytest.mark.parametrize("path", GOLDEN, ids=[os.path.basename(p)[:-4] for p in GOLDEN])
def test_oracle_matches_golden(path, oracle):
    z, tree, meta = load_case(path)
    q = z["q"]
    kinds = sorted({int(k[1]) for k in z.files if k.startswith("k") and k[1].isdigit()})
    assert kinds
    for kind in kinds:
        o = oracle.solve(tree, kind, q)
        for key in ("psw", "ptw_mid", "mid", "out"):
            assert rel(o[key], z[f"k{kind}_{key}"]) <= TOL, (kind, key, rel(o[key], z[f"k{kind}_{key}"]))
        if f"k{kind}_out_unfixed" in z.files:
            # all leaves on the last level: the reference's unmodified downward pass agrees
            assert rel(o["out"], z[f"k{kind}_out_unfixed"]) <= TOL
        m = z[f"k{kind}_direct"].shape[1]
        d = oracle.direct(meta["dim"], kind, meta["eps"], tuple(c[:m] for c in tree["targets"]), tree["sources"], q)
        assert rel(d, z[f"k{kind}_direct"]) <= 1e-14


def test_fix_matters_on_mixed_level_trees():
    """Where leaves sit above the last level the fixed downward pass differs
    from what the reference's loop bounds would compute; the golden case with
    mixed levels documents it (the reference's unmodified pass is not run there:
    it reads child index -1)."""
    z = np.load(os.path.join(HERE, "golden", "ref3d_plummer.npz"))
    assert int(z["last_level_only"][0]) == 0
    assert "k0_out_unfixed" not in z.files


def test_interp_basis_properties(oracle):
    rng = np.random.default_rng(0)
    for n in range(1, 13):
        lo, hi = -0.3, 1.7
        nodes = oracle.nodes(lo, hi, n)
        for x in rng.uniform(lo, hi, 20):
            b = oracle.interp_basis(x, lo, hi, n)
            assert abs(b.sum() - 1.0) < 1e-12  # partition of unity
            # reproduces polynomials of degree <= n
            for p in range(n + 1):
                assert abs(np.dot(b, nodes ** p) - x ** p) < 1e-10 * max(1.0, abs(x) ** p) * 10 ** (n / 4)
        # near-node branch: exact delta at (and within DBL_EPSILON of) a node
        for i in range(n + 1):
            b = oracle.interp_basis(nodes[i], lo, hi, n)
            assert b[i] == pytest.approx(1.0, abs=1e-12) and np.sum(np.abs(b)) == pytest.approx(1.0, abs=1e-12)


def test_reference_library_matches_golden(reflib):
    """Re-runs the reference library on one stored case (when it is built)."""
    z, tree, meta = load_case(os.path.join(HERE, "golden", "ref3d_plummer.npz"))
    rt = reflib.create(3, tree["targets"], degree=meta["deg"], cluster_size=meta["leaf"], theta=meta["theta"],
                       eps=meta["eps"])
    r = rt.solve(0, z["q"], fixed=True)
    assert rel(r["out"], z["k0_out"]) == 0.0


def test_oracle_field_kind_is_gradient(oracle):
    """FIELD = -grad_t of the potential: check by central differences."""
    rng = np.random.default_rng(4)
    for dim in (2, 3):
        src = tuple(rng.uniform(-1, 1, 50) for _ in range(dim))
        q = rng.uniform(-1, 1, 50)
        t = tuple(rng.uniform(2, 3, 5) for _ in range(dim))
        f = oracle.direct(dim, 2, 1e-3, t, src, q)
        h = 1e-5
        for d in range(dim):
            tp = tuple(c + (h if k == d else 0) for k, c in enumerate(t))
            tm = tuple(c - (h if k == d else 0) for k, c in enumerate(t))
            g = (oracle.direct(dim, 0, 1e-3, tp, src, q)[0] - oracle.direct(dim, 0, 1e-3, tm, src, q)[0]) / (2 * h)
            assert np.allclose(-g, f[1 + d], rtol=1e-6, atol=1e-9)
        assert np.allclose(f[0], oracle.direct(dim, 0, 1e-3, t, src, q)[0], rtol=1e-15)
