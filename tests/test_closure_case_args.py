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
