"""Host logic of the closure case runner: term-group gains and gain grids."""
import os
import sys

import pytest

sys.path.insert(0, os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "rast-3dmhd_b200"))
import closure_case  # noqa: E402


def test_term_gains():
    tg = closure_case.term_gains
    assert tg("stress+heat+emf") == {"stress": 1.0, "heat": 1.0, "emf": 1.0}
    assert tg("stress+heat+emf@0.12") == {"stress": 0.12, "heat": 0.12, "emf": 0.12}
    assert tg("stress@0.5+heat@0.25+emf@0") == {"stress": 0.5, "heat": 0.25, "emf": 0.0}
    assert tg("stress+heat@0.5+emf") == {"stress": 0.5, "heat": 0.5, "emf": 1.0}
    assert tg("emf") == {"emf": 1.0}
    with pytest.raises(ValueError):
        tg("stress+momentum")


def test_gain_grid():
    c = closure_case.gain_grid("stress+heat:0,0.25;emf:0,0.12")
    assert c == ["stress@0+heat@0+emf@0", "stress@0+heat@0+emf@0.12",
                 "stress@0.25+heat@0.25+emf@0", "stress@0.25+heat@0.25+emf@0.12"]
    assert closure_case.term_gains(c[3]) == {"stress": 0.25, "heat": 0.25, "emf": 0.12}


def test_eddy_factors():
    assert closure_case.eddy_factors("1,1.5,2:1:1.5") == [(1.0, 1.0, 1.0), (1.5, 1.5, 1.5), (2.0, 1.0, 1.5)]


def test_eddy_setup_scales_the_diffusion_coefficients():
    import mhd3d
    su = mhd3d.make_setup(mhd3d.convection_config(16, 16, 12))
    assert closure_case.eddy_setup(su, (1.0, 1.0, 1.0)) is su
    e = closure_case.eddy_setup(su, (2.0, 1.5, 3.0))
    p, q = su.params, e.params
    assert q.ore == p.ore * 2.0 and q.re == p.re / 2.0
    assert q.repr == p.repr / 1.5
    assert q.orm == p.orm * 3.0 and q.rm == p.rm / 3.0
    assert q.npx == p.npx and q.ocv == p.ocv and q.grav == p.grav
    assert e.grid is su.grid and e.state is su.state


def test_bias_candidates():
    c = closure_case.with_bias(closure_case.gain_grid("stress+heat:0,0.25;emf:0"))
    assert c == ["stress@0+heat@0+emf@0", "stress@0.25+heat@0.25+emf@0",
                 "stress@0+heat@0+emf@0|bias", "stress@0.25+heat@0.25+emf@0|bias"]   # the bias alone once
    assert closure_case.with_bias(["stress+heat+emf@0.5"])[-1] == "stress@0+heat@0+emf@0|bias"
    assert closure_case.split_bias("stress@0.06+heat@0.06+emf@0.12|bias") == ("stress@0.06+heat@0.06+emf@0.12", True)
    assert closure_case.split_bias("stress+heat+emf@0.12") == ("stress+heat+emf@0.12", False)
    assert closure_case.bias_alone("stress@0+heat@0+emf@0", True)
    assert not closure_case.bias_alone("stress@0+heat@0+emf@0", False)
    assert not closure_case.bias_alone("stress@0+heat@0+emf@0.12", True)
    assert closure_case.bias_alone("emf@0", True)   # groups not named take no network term


def test_residual_bias_is_the_mean_horizontal_profile():
    torch = pytest.importorskip("torch")
    g = torch.Generator().manual_seed(3)
    nz, ny, nx = 6, 5, 8
    prof = torch.randn(7, nz, 1, 1, generator=g, dtype=torch.float64)
    pairs = []
    for s in (1.0, 3.0):
        noise = torch.randn(7, nz, ny, nx, generator=g, dtype=torch.float64)
        noise -= noise.mean(dim=(2, 3), keepdim=True)
        pairs.append(((s * prof + noise).float(), None))
    b = closure_case.residual_bias(pairs)
    assert b.shape == (7, nz) and b.dtype == torch.float32
    assert torch.allclose(b.double(), 2.0 * prof[:, :, 0, 0], rtol=1e-5, atol=1e-6)
