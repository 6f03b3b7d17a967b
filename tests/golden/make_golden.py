"""Generate golden vectors by running the reference ``gradient_domain`` package.

Run once in a container that holds the reference sources:

    PYTHONDONTWRITEBYTECODE=1 python tests/golden/make_golden.py /root/reference

It imports ``gradient-domain/src`` from the given reference checkout, runs the
reference's own functions on small seeded inputs and writes
``tests/golden/golden.npz``.  The tests read only that file, so they run where
the reference is absent.
"""

from __future__ import annotations

import os
import sys

import numpy as np


def main(reference_root: str) -> None:
    sys.dont_write_bytecode = True
    sys.path.insert(0, os.path.join(reference_root, "gradient-domain", "src"))
    from gradient_domain import hdr, multigrid, operators, poisson, solvers, synthetic
    from gradient_domain.benchmark import manufactured_problem

    out: dict[str, np.ndarray] = {}

    # operators (operators.py:30-169)
    rng = np.random.default_rng(11)
    u = rng.standard_normal((23, 31))
    gx, gy = operators.gradient(u)
    out["op_u"], out["op_gx"], out["op_gy"] = u, gx, gy
    vx, vy = rng.standard_normal((23, 31)), rng.standard_normal((23, 31))
    out["op_vx"], out["op_vy"], out["op_div"] = vx, vy, operators.divergence(vx, vy)
    out["op_lap_h05"] = operators.laplacian(u, 0.5)
    ring = rng.standard_normal((14, 18))
    out["op_ring"], out["op_fold"] = ring, operators.fold_boundary(np.zeros((12, 16)), ring, 0.5)

    # one V-cycle from zero and from a nonzero iterate (multigrid.py:184-215)
    for name, shape, seed, opts, spacing in (
        ("vc63", (63, 63), 3, multigrid.MultigridOptions(), 1.0),
        ("vc47x61", (47, 61), 4, multigrid.MultigridOptions(pre_smoothing=1, post_smoothing=1), 1.0),
        ("vc30x22", (30, 22), 5, multigrid.MultigridOptions(pre_smoothing=3, post_smoothing=2), 0.5),
        ("vc8", (8, 8), 6, multigrid.MultigridOptions(), 1.0),
    ):
        b, _ = manufactured_problem(shape, seed=seed)
        u0 = np.random.default_rng(seed + 100).standard_normal(shape) * 0.1
        out[f"{name}_b"], out[f"{name}_u0"] = b, u0
        out[f"{name}_opts"] = np.array([opts.pre_smoothing, opts.post_smoothing,
                                        opts.coarsest_size, opts.coarsest_sweeps, spacing])
        out[f"{name}_zero"] = multigrid.v_cycle(np.zeros(shape), b, spacing, opts)
        out[f"{name}_warm"] = multigrid.v_cycle(u0, b, spacing, opts)

    # transfers (multigrid.py:169-181)
    fine = np.random.default_rng(6).standard_normal((31, 25))
    coarse = np.random.default_rng(7).standard_normal((15, 12))
    out["tr_fine"], out["tr_coarse"] = fine, coarse
    out["tr_restrict"] = multigrid._restrict(fine)
    out["tr_prolong"] = multigrid._prolong(coarse, (31, 25))

    # red-black Gauss-Seidel sweeps (multigrid.py:147-165), from float64 and float32 arrays
    for name, shape, sweeps, spacing in (("sm37x53", (37, 53), 1, 1.0),
                                         ("sm37x53s3", (37, 53), 3, 0.5),
                                         ("sm5x131", (5, 131), 2, 1.0),
                                         ("sm70x260s6", (70, 260), 6, 0.75)):
        rng = np.random.default_rng(sum(shape) + sweeps)
        u0, b = rng.standard_normal(shape), rng.standard_normal(shape)
        out[f"{name}_u0"], out[f"{name}_b"] = u0, b
        out[f"{name}_opts"] = np.array([sweeps, spacing])
        out[f"{name}_f64"] = multigrid._smooth(u0, b, spacing, sweeps)
        out[f"{name}_f32"] = multigrid._smooth(u0.astype(np.float32), b.astype(np.float32),
                                               spacing, sweeps)

    # multigrid.solve history (multigrid.py:218-255)
    b, _ = manufactured_problem((63, 63), seed=5)
    sol, rep = multigrid.solve(b, options=multigrid.MultigridOptions(tolerance=1e-10))
    out["mgsolve_b"], out["mgsolve_u"] = b, sol
    out["mgsolve_hist"] = np.array(rep.residuals)

    # every solver on the agreement case (tests/test_solvers.py:34-39)
    b, exact = manufactured_problem((47, 61), seed=4)
    out["sys_b"], out["sys_exact"] = b, exact
    for method in ("direct", "cg", "multigrid", "mgcg"):
        sol, rep = solvers.solve_system(b, method=method, tolerance=1e-10)
        out[f"sys_{method}_u"] = sol
        out[f"sys_{method}_info"] = np.array([rep.iterations, rep.relative_residual,
                                              float(rep.converged)])

    # Neumann DCT solver (solvers.py:224-262)
    for shape, seed in (((32, 40), 9), ((97, 131), 8), ((64, 64), 12)):
        bb = np.random.default_rng(seed).standard_normal(shape)
        bb -= bb.mean()
        key = f"neu{shape[0]}x{shape[1]}"
        out[f"{key}_b"], out[f"{key}_u"] = bb, solvers.solve_neumann(bb)

    # application entry points (poisson.py, hdr.py)
    img = np.random.default_rng(0).random((40, 52, 3))
    yy, xx = np.mgrid[0:40, 0:52]
    disc = (yy - 20.0) ** 2 + (xx - 26.0) ** 2 < 14.0 ** 2
    src = np.random.default_rng(1).random((40, 52, 3))
    field = poisson.GuidanceField.of(src)
    out["app_img"], out["app_src"], out["app_disc"] = img, src, disc
    out["app_masked"] = poisson.solve_masked(field, img, disc)[0]
    out["app_dirichlet"] = poisson.solve_dirichlet(field, img, method="direct")[0]

    ex = synthetic.make_compositing_example(shape=(96, 144), seed=0)
    out["clone_target"], out["clone_source"] = ex.target, ex.source
    out["clone_mask"], out["clone_offset"] = ex.mask, np.array(ex.offset)
    for mode in ("import", "mixed", "average"):
        out[f"clone_{mode}_mask"] = poisson.seamless_clone(
            ex.source, ex.target, ex.mask, ex.offset, mode=mode, domain="mask")[0]
    out["clone_import_rect"] = poisson.seamless_clone(
        ex.source, ex.target, ex.mask, ex.offset, domain="rectangle", method="direct")[0]

    tex, edges = synthetic.make_texture_example(shape=(48, 56), seed=1)
    out["tex_image"], out["tex_edges"] = tex, edges
    out["tex_flat"] = poisson.texture_flatten(tex, edges, method="direct")[0]
    ty, tx = np.mgrid[0:48, 0:56]
    illum_mask = (ty - 24.0) ** 2 + (tx - 28.0) ** 2 < 15.0 ** 2
    out["illum_mask"] = illum_mask
    out["illum"] = poisson.illumination_change(tex, illum_mask, alpha=0.4, beta=0.6)[0]

    rad = synthetic.make_radiance_map(shape=(48, 64), seed=2)
    out["tm_radiance"] = rad
    mapped, factor = hdr.tone_map(rad)
    out["tm_mapped"], out["tm_factor"] = mapped, factor
    lum = np.log(np.maximum(rad @ np.array([0.2126, 0.7152, 0.0722]), np.finfo(float).tiny))
    out["att_levels1"] = hdr.attenuation_field(lum, hdr.ToneMapConfig(alpha=0.1, beta=0.85,
                                                                      levels=1))

    path = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden.npz")
    np.savez_compressed(path, **out)
    print(f"wrote {path}: {len(out)} arrays, {os.path.getsize(path) / 1024:.0f} KiB")


def suite(reference_root: str) -> None:
    """Inputs of the reference's own test suite (gradient-domain/tests), made by the
    reference's procedural image generators (synthetic.py), written to suite.npz.

    tests/test_reference_suite.py re-runs every case of test_solvers.py,
    test_operators.py and test_applications.py on these inputs through the B200
    package; the generators themselves are test data, not part of the solve path.
    """
    sys.dont_write_bytecode = True
    sys.path.insert(0, os.path.join(reference_root, "gradient-domain", "src"))
    from gradient_domain import synthetic
    from gradient_domain.benchmark import manufactured_problem

    out: dict[str, np.ndarray] = {}
    # test_applications.py:32-34 (module fixture)
    ex = synthetic.make_compositing_example(shape=(160, 240), seed=0)
    out["ex_target"], out["ex_source"] = ex.target, ex.source
    out["ex_mask"], out["ex_offset"] = ex.mask, np.array(ex.offset)
    out["ex_naive"] = ex.naive_composite()
    # test_applications.py:149-164
    for shape in ((96, 96), (128, 128)):
        image, edges = synthetic.make_texture_example(shape=shape, seed=1)
        out[f"tex{shape[0]}_image"], out[f"tex{shape[0]}_edges"] = image, edges
    # test_applications.py:178-198
    for shape in ((128, 176), (96, 128)):
        out[f"rad{shape[0]}x{shape[1]}"] = synthetic.make_radiance_map(shape=shape, seed=2)
    # the manufactured right-hand sides the solver tests draw (test_solvers.py), to pin
    # this package's restatement of benchmark.manufactured_problem
    for shape, seed in (((63, 63), 3), ((47, 61), 4), ((127, 127), 7), ((33, 33), 10),
                        ((31, 31), 5)):
        out[f"mp{shape[0]}x{shape[1]}s{seed}"] = manufactured_problem(shape, seed=seed)[0]
    path = os.path.join(os.path.dirname(os.path.abspath(__file__)), "suite.npz")
    np.savez_compressed(path, **out)
    print(f"wrote {path}: {len(out)} arrays, {os.path.getsize(path) / 1024:.0f} KiB")


if __name__ == "__main__":
    args = [a for a in sys.argv[1:] if not a.startswith("--")]
    root = args[0] if args else "/root/reference"
    if "--suite" not in sys.argv:
        main(root)
    suite(root)
