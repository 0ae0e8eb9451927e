"""Full-size parity of the assembly against the oracle: sampled rows of whole
benchmark systems (the 400x120 layered mesh, the 300x150 jittered mesh, the
600x200 jittered mesh with topography and a 4-element strip).

The oracle integrates only the elements that touch the sampled rows
(orc_asmble_rows: the same arithmetic and element order as its full
ASMBLE_DRIVER restatement), so whole systems of 2.2-5.8 M DOF are checked
row by row.  Rows cover every DOF class (PML, Bielak strip, interior, strip
boundary), free-surface rows (topography included) and the first and last
rows.  Tolerances:
  * batched affine assembly (complex128 ring slot) vs oracle FP64:  <= 1e-12
    per row (max |a - ref| / max |ref row|)
  * plain FP64 assembly vs oracle FP64:                            bit-identical
  * ASMBLE_DRIVER COMPLEX*8 CDIST (host buffer) vs the oracle's
    FP32 cast-then-add accumulation:                                 bit-identical
The sparsity of the product graph is checked against the oracle's graph of
the same mesh first (bit-exact)."""
import numpy as np
import pytest

import oracle
from fem25_b200 import Context, graph_build, synth
from tests import helpers

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu


def _dev():
    return torch.device("cuda:0")


# systems checked per configuration: indices into the configuration's
# (f, py) list -- the lowest and highest frequency, ky = 0 and the largest ky
_SYSTEMS = {1: [0, 300, 511], 3: [95, 1151], 4: [0, 2500, 4799]}


@pytest.mark.parametrize("cfg", [1, 3, 4])
def test_fullsize_rows_match_oracle(cfg):
    mesh, pairs, _ = synth.make_config(cfg)
    g = graph_build(mesh)
    go = oracle.graph_build(mesh)
    for k in ("lm", "irptr", "jcptr", "cnp"):
        assert np.array_equal(getattr(g, k), getattr(go, k)), k
    del go
    rows = helpers.sample_rows(mesh, g, per_class=12, seed=cfg)
    sel = _SYSTEMS[cfg]
    ctx = Context(mesh, g)
    dev = _dev()
    nz = ctx.nzero
    try:
        # batched assembly of the selected systems into a ring of len(sel)
        # 128-byte aligned complex128 slots
        sst = (2 * nz + 15) // 16 * 16
        ring = torch.empty(len(sel) * sst, dtype=torch.float64, device=dev)
        ctx.assemble_batch("B", [pairs[k][0] for k in sel], [pairs[k][1] for k in sel], ring, sst,
                           len(sel))
        torch.cuda.synchronize()
        plain = torch.empty(nz, dtype=torch.complex128, device=dev)
        worst = 0.0
        for slot, k in enumerate(sel):
            f, py = pairs[k]
            idx, r128, r64 = oracle.asmble_rows(mesh, g, rows, "B", f, py)
            ti = torch.from_numpy(idx).to(dev)
            b = ring[slot * sst:slot * sst + 2 * nz].view(-1, 2)[ti].cpu().numpy()
            err = helpers.rows_err(b[:, 0] + 1j * b[:, 1], r128, idx, g, rows)
            worst = max(worst, err)
            assert err <= 1e-12, (cfg, k, err)
            # plain FP64 path: bit-identical
            ctx.assemble("B", f, py, plain, None)
            torch.cuda.synchronize()
            p = plain[ti].cpu().numpy()
            assert np.array_equal(p, r128), (cfg, k, "plain FP64 rows differ")
        del ring, plain
        torch.cuda.empty_cache()
        # ASMBLE_DRIVER drop-in with a host buffer, COMPLEX*8 bit-identical
        f, py = pairs[sel[-1]]
        idx, _, r64 = oracle.asmble_rows(mesh, g, rows, "S", f, py)
        cdist = ctx.asmble_driver("S", f, py)
        assert np.array_equal(cdist[idx].view(np.uint32), r64.view(np.uint32)), cfg
        print(f"config {cfg}: {len(rows)} rows, {len(idx)} entries per system, "
              f"batched max row error {worst:.2e}")
    finally:
        ctx.close()
        torch.cuda.empty_cache()
