"""Sparsity at the benchmark sizes: the library's graph set-up
(fem25_graph_build) against the oracle's GENIEN -> GENID -> GENLM ->
CONNECT -> GENCRS_QUICK -> CNMESH restatement (graph25_driver.f90:2-72) on
the 400x120 layered mesh, the 300x150 jittered mesh and the 600x200
jittered mesh with topography.  IEN, LM, IRPTR, JCPTR and CNP must be
identical (integer work: bit-exact)."""
import numpy as np
import pytest

import oracle
from fem25_b200 import graph_build, synth


@pytest.mark.parametrize("cfg", [1, 3, 4])
def test_fullsize_graph_matches_oracle(cfg):
    mesh, _, _ = synth.make_config(cfg)
    g = graph_build(mesh)
    go = oracle.graph_build(mesh)
    assert (g.ndof, g.nzero) == (go.ndof, go.nzero)
    for k in ("ien", "lm", "irptr", "jcptr", "cnp"):
        assert np.array_equal(getattr(g, k), getattr(go, k)), k
