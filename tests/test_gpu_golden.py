"""The CUDA engine against the reference's own outputs (golden fixtures made
by the reference cuSPARSE driver) and against the oracle on the same inputs."""
import numpy as np
import pytest

from oracle import oracle

from golden_util import assert_matches_reference, cases
from helpers import assert_parity

pytestmark = pytest.mark.gpu

GOLDEN = cases()


@pytest.mark.parametrize("algo", ["plain", "learned", "cusparse"])
@pytest.mark.parametrize("name,A,B,C", GOLDEN, ids=[g[0] for g in GOLDEN])
def test_engine_matches_reference_outputs(engine, name, A, B, C, algo):
    got, rep = engine.multiply(A, B, algo=algo)
    H = got.to_host()
    R = oracle.spgemm(A, B)
    assert_matches_reference(H, C, R.bound)
    if algo != "cusparse":
        assert_parity(H, R)  # and bit-exact with the canonical-order oracle
