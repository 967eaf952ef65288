"""Collocation-matrix assembly on the GPU against the oracle's rows."""
import numpy as np
import pytest

import oracle
from bielcc_b200 import abi
from bielcc_b200 import workloads as W
from conftest import TOL_FP64, TOL_MIXED, rel_l2

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("layout", [abi.LAYOUT_TAU2, abi.LAYOUT_FULL3])
def test_assemble_tri320(gctx, layout):
    cells = W.perturbed_icosphere(level=2, seed=2)
    k = 4 * np.pi
    m = gctx.mesh(cells)
    A, rep = gctx.assemble_K(m, k, layout=layout)
    Ao = oracle.assemble_K(cells, k, layout=layout)
    assert rep.n_near_pairs > len(cells)
    assert rel_l2(A, Ao) < TOL_FP64
    Am, _ = gctx.assemble_K(m, k, layout=layout, c64=True, precision="mixed")
    assert Am.dtype == np.complex64
    assert rel_l2(Am.astype(np.complex128), Ao) < TOL_MIXED


def test_assemble_quads_complex_k_adaptive(gctx):
    cells = W.uv_sphere(6, 12)
    m = gctx.mesh(cells)
    for npm in (abi.NumParam.default(), abi.NumParam.default(n_start=4, n_start_seg=6, p_max=2, p_max_seg=2),
                abi.NumParam.default(n_start=4, n_start_seg=6, p_max=3, p_max_seg=2)):
        A, _ = gctx.assemble_K(m, complex(3.0, 0.2), numparam=npm)
        Ao = oracle.assemble_K(cells, complex(3.0, 0.2), numparam=npm)
        assert rel_l2(A, Ao) < TOL_FP64


@pytest.mark.parametrize("p_max,eps", [(3, None), (4, None), (3, 1e-14), (4, 1e-14), (3, 1e3)])
def test_assemble_adaptive_per_column(gctx, p_max, eps):
    """p_max >= 3: every far block's column test at the second pass. Columns
    that pass take the pass at 2 n_start, failing ones the pass at 4 n_start
    (p_max = 3) or the whole loop (p_max = 4). Default eps (a mix of both),
    eps = 1e-14 (every column fails), eps = 1e3 (none fails); both layouts,
    triangles, complex k; FP64 against the oracle's loop, mixed within the
    mixed tolerance."""
    cells = W.perturbed_icosphere(level=1, seed=7)
    m = gctx.mesh(cells)
    k = complex(3.0, 0.2)
    npm = abi.NumParam.default(n_start=3, n_start_seg=4, p_max=p_max, p_max_seg=2)
    if eps is not None:
        npm.eps = eps
    for layout in (abi.LAYOUT_TAU2, abi.LAYOUT_FULL3):
        A, _ = gctx.assemble_K(m, k, numparam=npm, layout=layout)
        Ao = oracle.assemble_K(cells, k, numparam=npm, layout=layout)
        assert rel_l2(A, Ao) < TOL_FP64
        Am, _ = gctx.assemble_K(m, k, numparam=npm, layout=layout, precision="mixed")
        assert rel_l2(Am, Ao) < TOL_MIXED


def test_assemble_large_rows_sample(gctx):
    """A 5120-triangle icosphere: sampled rows against the oracle."""
    cells = W.perturbed_icosphere(level=4, seed=2)
    m = gctx.mesh(cells)
    A, _ = gctx.assemble_K(m, 4 * np.pi, c64=True, precision="mixed")
    for r0 in (0, 2000, 5100):
        Ao = oracle.assemble_K(cells, 4 * np.pi, rows=(r0, r0 + 8))
        assert rel_l2(A[2 * r0: 2 * r0 + 16].astype(np.complex128), Ao) < TOL_MIXED
