"""Mirror-symmetry and extrusion filters composed with the smoothing filter
(pyto_symmetry_filter + pyto_filter) against the reference's matrices
(tests/golden/sym_filters.npz, from PyTO's createFilters)."""
import types

import numpy as np
import pytest
import scipy.sparse as sp
import torch

import oracle as O
from conftest import golden

pytestmark = pytest.mark.gpu

CASES = [("a", (7, 5, 4), (1.0, 1.0, 1.0)), ("b", (6, 3, 5), (1.0, 0.5, 2.0))]


def _ref(d, tag, name, ne):
    return sp.coo_matrix((d[f"{tag}_{name}_val"], (d[f"{tag}_{name}_row"], d[f"{tag}_{name}_col"])),
                         shape=(ne, ne)).tocsr()


def _mesh(nel, h):
    from pyto_b200.hex_mesher import HexMesher
    m = HexMesher()
    m.grid_mesh(nel, h)
    return m


@pytest.mark.parametrize("tag,nel,h", CASES)
def test_single_maps_match_reference(tag, nel, h):
    from pyto_b200 import topopt_filters as tf
    d = golden("sym_filters.npz")
    m = _mesh(nel, h)
    ne = int(np.prod(nel))
    x = np.random.default_rng(0).uniform(0.01, 1.0, ne)
    for name, fn in (("mx", tf.createXSymmetryFilter), ("my", tf.createYSymmetryFilter),
                     ("mz", tf.createZSymmetryFilter), ("ex", tf.createXExtrudeFilter),
                     ("ey", tf.createYExtrudeFilter), ("ez", tf.createZExtrudeFilter)):
        F = fn(m)
        np.testing.assert_allclose(F @ x, _ref(d, tag, name, ne) @ x, rtol=1e-14, atol=1e-15, err_msg=name)


@pytest.mark.parametrize("tag,nel,h", CASES)
def test_composed_filter_matches_create_filters(tag, nel, h):
    from pyto_b200 import topopt_common as tc
    d = golden("sym_filters.npz")
    m = _mesh(nel, h)
    ne = int(np.prod(nel))
    params = tc.TOParams(RelativeFilterRadius=1.5, XSymmetry=True, ZSymmetry=True, ExtrudeY=True)
    H, Hs = tc.createFilters(types.SimpleNamespace(mesh=m), params)
    Href = _ref(d, tag, "all", ne)
    np.testing.assert_allclose(Hs, d[f"{tag}_all_Hs"], rtol=1e-13)
    rng = np.random.default_rng(1)
    x = rng.uniform(0.05, 1.0, ne)
    g = -rng.uniform(0.1, 1.0, ne)
    np.testing.assert_allclose(H @ x, Href @ x, rtol=1e-13, atol=1e-15)
    np.testing.assert_allclose(H.T @ g, Href.T @ g, rtol=1e-13, atol=1e-15)
    np.testing.assert_allclose(H.density(x), (Href @ x) / Hs, rtol=1e-13)
    np.testing.assert_allclose(H.chain(g), Href.T @ (g / Hs), rtol=1e-13, atol=1e-15)
    np.testing.assert_allclose(H.sensitivity(g, x), (Href @ (x * g)) / Hs / x, rtol=1e-13)
    dens = H.density(torch.as_tensor(x, device="cuda"))
    assert isinstance(dens, torch.Tensor) and dens.is_cuda
