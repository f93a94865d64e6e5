"""The relabelled CSR every counting kernel reads (Graph.view /
beep_graph_view) against the oracle's peel and priority order, entry for
entry: rows of every size class of the row sort, hub rows of several
thousand to ~50,000 entries whose tiles go through up to four merge passes,
both orders and several peel thresholds."""
import numpy as np
import pytest

import beep_b200 as B
from oracle import pyoracle as O
from oracle import synth


def hub_graph(n, hub_degrees, p_background, seed):
    """ER background plus hubs 0.. with the given degrees to random vertices."""
    rng = np.random.default_rng(seed)
    rp, col = synth.erdos_renyi(n, p_background, seed)
    src = np.repeat(np.arange(n, dtype=np.int64), np.diff(rp))
    us, vs = [src], [col.astype(np.int64)]
    for h, d in enumerate(hub_degrees):
        nb = rng.choice(np.arange(len(hub_degrees), n), size=d, replace=False)
        us.append(np.full(d, h, dtype=np.int64))
        vs.append(nb.astype(np.int64))
    return synth.to_csr(n, np.concatenate(us), np.concatenate(vs))


def graphs():
    yield "er", synth.erdos_renyi(3000, 0.004, 5)
    yield "er_sparse", synth.erdos_renyi(5000, 0.0005, 6)  # rows of 1 and 2 entries
    yield "rmat14", synth.rmat(14, 16, 0.57, 0.19, 0.19, 3)
    yield "chung_lu", synth.chung_lu(1 << 15, 48.0, 2.0, 9)
    # hub rows of 4097 .. 50,000 entries: 2 .. 13 tiles of 4096
    yield "hubs", hub_graph(1 << 16, [4097, 4096, 8192, 8193, 12300, 20000, 50000], 6.0 / (1 << 16), 21)


@pytest.mark.gpu
@pytest.mark.parametrize("name,csr", list(graphs()), ids=lambda x: x if isinstance(x, str) else "")
def test_view_equals_oracle(ctx, name, csr):
    rp, col = csr
    g = B.Graph.from_csr(ctx, rp, col)
    for min_qdeg in (1, 2, 3, 5):
        for asc in (True, False):
            got = g.view(min_qdeg, asc)
            exp = O.view(rp, col, min_qdeg, asc)
            for what, a, b in zip(("row_ptr", "col", "orig"), got, exp):
                assert np.array_equal(a, b), (name, min_qdeg, asc, what)
    g.close()
