"""Known-answer tests of the walk's physics on the CPU restatement (which
the golden fixtures pin to the reference): energy bookkeeping.  Every
quantum of every photon's start weight is absorbed, leaves through the top
or the bottom, is still held at the 10,000-step cap, or is removed / added
by roulette; the only other change is the rounding of the float weight in
`w - w_t`, tracked exactly.  In FP64 that rounding is zero."""
import pytest

from conftest import CONFIGS

import oracle


def load_case(case):
    """The case's configuration read by the oracle's own reader (these tests
    need no part of the CUDA library)."""
    d = CONFIGS / case
    return oracle.read_config(d / "sim_set.json", d / "input.txt")[0]


def balance(e):
    return (e["start"] + e["roulette_gained"] + e["rounding"]
            - e["absorbed"] - e["top"] - e["bottom"] - e["capped"] - e["roulette_lost"])


@pytest.mark.parametrize("case", ["fiber3", "ring5", "mismatch", "three_layer"])
@pytest.mark.parametrize("roulette", [True, False])
def test_energy_is_conserved(case, roulette):
    sim = load_case(case)
    e = oracle.energy(sim, 400, 7, roulette=roulette)
    assert balance(e) == 0.0, e
    assert e["absorbed"] > 0 and e["top"] > 0
    if not roulette:
        assert e["roulette_lost"] == 0 and e["roulette_gained"] == 0
    e64 = oracle.energy(sim, 400, 7, fp64=True, roulette=roulette)
    assert e64["rounding"] == 0.0 and balance(e64) == 0.0, e64
