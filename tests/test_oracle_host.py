"""Host-side checks of the oracle's own machinery (CPU only): its checkpoint of the dynamic
state, and its row-parallel connect(p) against a direct restatement of the draw."""
import numpy as np

from brian2cuda_b200 import models

DT = 1e-4
mV = 1e-3


def _delay_net(net, n=400, seed=3):
    rng = np.random.default_rng(seed)
    G = net.lif_group(n, models.cuba_lif(), "float64")
    net.set_state(G, "v", rng.uniform(-60 * mV, -50 * mV, n))
    i, j = models.bernoulli_pairs(rng, n, n, 0.05)
    d = rng.integers(1, 17, size=len(i)).astype(np.int32)
    exc = i < int(0.8 * n)
    Ce = net.synapses(G, G, "ge", i[exc], j[exc], w_scalar=1.62 * mV, delay=d[exc])
    net.synapses(G, G, "gi", i[~exc], j[~exc], w_scalar=-9 * mV, delay=d[~exc])
    return G, Ce


def test_oracle_store_restore_replays_identically(oracle_factory):
    """Runs from one checkpoint give the same spikes, state and delay queue, also with
    spikes in flight at the checkpoint."""
    net = oracle_factory(DT)
    G, Ce = _delay_net(net)
    net.run(97)
    net.store(0)
    q0 = net.queue(Ce)
    assert len(q0) > 0
    res = []
    for _ in range(2):
        net.restore(0)
        assert net.timestep == 97
        np.testing.assert_array_equal(net.queue(Ce), q0)
        net.run(120)
        idx, st = net.spikes(G)
        keep = st >= 97
        res.append((idx[keep], st[keep], net.get_state(G, "v"), net.queue(Ce)))
    # the monitor keeps both runs' records: the second run's spikes appear twice
    idx2, st2 = res[1][0], res[1][1]
    first = res[0]
    assert len(idx2) == 2 * len(first[0]) and len(first[0]) > 50
    order = np.lexsort((first[0], first[1]))
    np.testing.assert_array_equal(np.sort(st2)[::2], first[1][order])
    np.testing.assert_array_equal(res[1][2], first[2])
    np.testing.assert_array_equal(res[1][3], first[3])


def test_oracle_connect_matches_direct_draw():
    """The oracle's row-parallel connect(p) equals the draw restated row by row in numpy:
    pair (i, j) connects when word j mod 4 of Philox(j/4, i, 0x5EED, 0) is below p 2^32,
    and rows list their synapses by delay, then j."""
    from oracle.oracle import OracleNet

    from _philox import philox4x32_10
    net = OracleNet(DT)
    A = net.lif_group(37, models.cuba_lif())
    B = net.lif_group(53, models.cuba_lif())
    seed, p, dmin, dmax = 0xABCDEF0123, 0.3, 2, 9
    sid = net.synapses_random(A, B, "ge", p, dmin, dmax, 1e-3, seed, pre_range=(5, 30))
    got = [net.syn_get(sid, v) for v in ("i", "j", "delay")]
    thr = int(p * 4294967296.0)
    k0, k1 = seed & 0xFFFFFFFF, seed >> 32
    I, J, D = [], [], []
    for i in range(5, 30):
        row = []
        for jq in range((53 + 3) // 4):
            w = philox4x32_10((jq, i, 0x5EED, 0), (k0, k1))
            for e in range(4):
                j = 4 * jq + e
                if j < 53 and w[e] < thr:
                    wd = philox4x32_10((j, i, 0xDE1A, 1), (k0, k1))
                    row.append((dmin + ((wd[0] * (dmax - dmin + 1)) >> 32), j))
        row.sort(key=lambda x: x[0])         # stable: j order within a delay
        for d, j in row:
            I.append(i)
            J.append(j)
            D.append(d)
    np.testing.assert_array_equal(got[0], I)
    np.testing.assert_array_equal(got[1], J)
    np.testing.assert_array_equal(got[2], D)
    assert len(I) > 100
