"""The drop-in boundary end to end: the reference's unmodified FvMatrix / fvm::laplacian code, with
its cfd::solveLdu calls redirected at link time to the GPU library through
include/voluma_b200_ldu.hpp (oracle/dropin_driver.cpp).  In CFD_REPRODUCIBLE mode the result must
equal the reference's own all-CPU run bit for bit; with GAMG it must reach the same tolerance."""
import numpy as np
import pytest

from conftest import load_golden
from oracle import ref

pytestmark = [pytest.mark.gpu, pytest.mark.skipif(not ref.dropin_available(), reason="drop-in library not built")]


def spec(g):
    return dict(lo=tuple(g["spec_lo"]), hi=tuple(g["spec_hi"]), periodic=tuple(g["spec_periodic"]),
                points=g.get("points"))


@pytest.mark.parametrize("name", ["jitter10x8x6", "periodic8", "walls7x5x3"])
def test_reference_code_with_gpu_solveLdu_is_bitwise(name):
    g = load_golden(name)
    if g["spec_beta"].any() and "points" not in g:
        pytest.skip("stretched spec is reproduced through points only")
    p, flux, perf, calls = ref.dropin_pressure_solve(tuple(g["spec_n"]), g["ps_gamma"], g["ps_divphi"],
                                                     np.zeros(g["n_cells"]), n_non_orth=2, grad_scheme=1,
                                                     precond="diagonal", max_iter=3000, reproducible=True, **spec(g))
    assert calls == 3
    assert np.array_equal(p, g["ps_p"])
    assert np.array_equal(flux, g["ps_flux"])
    assert np.array_equal(perf[:, 4], g["ps_perf"][:, 4])


@pytest.mark.parametrize("name", ["jitter10x8x6", "periodic24"])
def test_reference_code_with_gpu_gamg(name):
    g = load_golden(name)
    p, flux, perf, calls = ref.dropin_pressure_solve(tuple(g["spec_n"]), g["ps_gamma"], g["ps_divphi"],
                                                     np.zeros(g["n_cells"]), n_non_orth=2, grad_scheme=1,
                                                     precond="GAMG", max_iter=500, **spec(g))
    assert calls == 3 and perf[:, 5].all()
    assert np.linalg.norm(p - g["ps_p"]) <= 1e-5 * np.linalg.norm(g["ps_p"])
