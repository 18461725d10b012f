"""The a posteriori closure case end to end at a tiny size: two fine FP64 runs,
commutator training and residual fine-tuning, the gain chosen on the training
run's window, coarse runs scored against the filtered fine profiles, and the
saved case reloaded (the plain coarse run must come out the same)."""
import math
import os
import sys

import pytest

from test_gpu_parity import _gpu_or_skip

pytestmark = pytest.mark.gpu

ARGS = ["--fine", "64", "64", "32", "--ra", "1e5", "--ta", "1e4", "--contrast", "3", "--spin", "0.02",
        "--settle", "0.01", "--window", "0.06", "--samples", "3", "--chunk", "50", "--iters", "30",
        "--resid-steps", "2", "--resid-iters", "30", "--gains", "1,0.5", "--bias"]


def test_closure_case_small(mhd3d, tmp_path):
    _gpu_or_skip(mhd3d)
    pytest.importorskip("torch")
    sys.path.insert(0, os.path.dirname(mhd3d.__file__))
    import closure_case
    saved = str(tmp_path / "case.npz")
    res = closure_case.main(ARGS + ["--save", saved])
    assert res["fine"] == [64, 64, 32]
    assert res["window"][1] > res["window"][0]
    assert 0 < res["settle"] < 0.02   # the coarse runs start from the filtered state before the window
    assert res["train"]["pairs"] == 4 and res["train"]["residual"]["pairs"] == 4
    assert set(res["a_priori"]) == {"commutator_error_ratio", "residual_error_ratio", "commutator_vs_residual_ratio",
                                    "bias_residual_error_ratio", "network_and_bias_residual_error_ratio"}
    assert res["train"]["gain_chosen"] in ("stress+heat+emf@1", "stress+heat+emf@0.5", "stress+heat+emf@1|bias",
                                           "stress+heat+emf@0.5|bias", "stress@0+heat@0+emf@0|bias")
    names = [k for k in res if k == "plain" or k.startswith("closure")]
    assert "plain" in names and len(names) >= 3   # plain, the default variant, the chosen gain
    for k in names:
        run = res[k]
        assert run["status"] == 0, (k, run)
        assert all(math.isfinite(v) for v in run["profile_rel_err"].values()), (k, run)
        if k != "plain":
            # the bias alone evaluates no network
            evals = 0 if run["closure"]["bias_only"] else run["steps"]
            assert run["closure"]["evals"] == evals and run["closure"]["err"] == 0
    # the reloaded case starts the coarse runs from the same filtered state
    again = closure_case.main(ARGS + ["--load", saved, "--variants", ""])
    assert again["plain"]["profile_rel_err"] == res["plain"]["profile_rel_err"]
    assert again["plain"]["steps"] == res["plain"]["steps"]
