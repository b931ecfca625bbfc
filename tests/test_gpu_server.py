"""Ray-query server: every request gets the same result alone (plain path, one
launch per request) and in the mix (coalesced with other scenes' requests in
shared launches); updates are ordered; admission respects the HBM budget."""
import numpy as np
import pytest

import oracle
from shinobi_b200 import scenes

pytestmark = pytest.mark.gpu


def _scene_set():
    return [scenes.uniform_soup(n, seed=40 + i, offset_scale=s)
            for i, (n, s) in enumerate([(3000, 0.02), (20000, 0.005), (500, 0.05), (60000, 0.002)])]


def _rays8(n, seed, tmax):
    o, d = scenes.random_rays(n, seed=seed)
    r = np.zeros((n, 8), np.float32)
    r[:, 0:3] = o
    r[:, 3:6] = d
    r[:, 6] = tmax
    return r


def _requests(shn, nreq=40):
    rng = np.random.default_rng(5)
    out = []
    for k in range(nreq):
        n = int(rng.integers(100, 20000))
        kind = shn._abi.SHN_REQ_CLOSEST if k % 2 == 0 else shn._abi.SHN_REQ_ANY
        tmax = 1e30 if kind == shn._abi.SHN_REQ_CLOSEST else 0.3
        out.append((kind, k % 4, _rays8(n, 1000 + k, tmax)))
    return out


def _run(srv, reqs, sequential):
    outs = []
    tickets = []
    for kind, slot, rays in reqs:
        tri = np.zeros(rays.shape[0], np.uint32)
        t = np.zeros(rays.shape[0], np.float32)
        outs.append((tri, t))
        r = srv.ray_request(kind, slot, rays, tri, t)
        tk = srv.submit(r)
        if sequential:
            assert srv.wait(tk) == 0
        else:
            tickets.append(tk)
    for tk in tickets:
        assert srv.wait(tk) == 0
    return outs


def _oracle(sc, rays, kind):
    b = oracle.bounds(sc.vertices, sc.indices)
    g = oracle.build_uniform(sc.vertices, sc.indices, b, oracle.resolution(sc.num_triangles, b, 5.0))
    if kind == 0:
        tri, t, _, _, _ = oracle.trace_closest(g, rays[:, 0:3], rays[:, 3:6], rays[:, 6])
        return tri, t
    occ, _ = oracle.trace_any(g, rays[:, 0:3], rays[:, 3:6], rays[:, 6])
    return occ, None


def test_same_result_alone_and_in_the_mix(gpu):
    import shinobi_b200 as shn
    scs = _scene_set()
    reqs = _requests(shn)
    plain = shn.Server(coalesce=False, num_slots=4)
    mixed = shn.Server(coalesce=True, num_slots=4)
    for i, sc in enumerate(scs):
        plain.load_scene(i, sc)
        mixed.load_scene(i, sc)
    a = _run(plain, reqs, sequential=True)
    b = _run(mixed, reqs, sequential=False)
    for (ta, xa), (tb, xb) in zip(a, b):
        assert np.array_equal(ta, tb)
        assert np.array_equal(xa.view(np.uint32), xb.view(np.uint32))
    st_plain, st_mix = plain.stats(), mixed.stats()
    assert st_plain["launches"] == len(reqs)
    assert st_mix["launches"] < len(reqs)          # requests were coalesced
    assert st_mix["max_requests_per_launch"] > 1
    # and the results are the oracle's
    for k in (0, 1, 6, 7):
        kind, slot, rays = reqs[k]
        ref, reft = _oracle(scs[slot], rays, kind)
        if kind == 0:
            assert np.array_equal(b[k][0], ref)
            assert np.array_equal(b[k][1].view(np.uint32), reft.view(np.uint32))
        else:
            assert np.array_equal((b[k][0] != shn.SHN_MISS).astype(np.uint8), ref)
    plain.close()
    mixed.close()


def test_updates_are_ordered(gpu):
    import shinobi_b200 as shn
    A = scenes.uniform_soup(5000, seed=1, offset_scale=0.02)
    B = scenes.uniform_soup(5000, seed=2, offset_scale=0.02)
    srv = shn.Server(num_slots=2)
    srv.load_scene(0, A)
    rays = _rays8(8000, 9, 1e30)
    out1 = (np.zeros(8000, np.uint32), np.zeros(8000, np.float32))
    out3 = (np.zeros(8000, np.uint32), np.zeros(8000, np.float32))
    t1 = srv.submit(srv.ray_request(0, 0, rays, *out1))
    t2 = srv.submit(srv.update_request(0, B))
    t3 = srv.submit(srv.ray_request(0, 0, rays, *out3))
    assert srv.wait(t1) == 0 and srv.wait(t2) == 0 and srv.wait(t3) == 0
    ra, _ = _oracle(A, rays, 0)
    rb, _ = _oracle(B, rays, 0)
    assert np.array_equal(out1[0], ra)
    assert np.array_equal(out3[0], rb)
    assert srv.stats()["updates"] == 1
    srv.close()


@pytest.mark.parametrize("coalesce", [True, False])
def test_repeated_replacements_of_one_slot(gpu, coalesce):
    """A slot replaced again and again, by scenes larger and smaller than the
    one before (each replacement rebuilds into the buffers the slot released
    last time, growing them where needed): every request sees the scene of its
    turn, and the slot left alone keeps its own."""
    import shinobi_b200 as shn
    seq = [scenes.uniform_soup(n, seed=70 + i, offset_scale=0.01)
           for i, n in enumerate([4000, 12000, 2500, 12000, 4000, 9000])]
    other = scenes.uniform_soup(3000, seed=90, offset_scale=0.02)
    srv = shn.Server(num_slots=2, coalesce=coalesce)
    srv.load_scene(0, seq[0])
    srv.load_scene(1, other)
    rays = _rays8(6000, 21, 1e30)
    outs = []
    for k in range(len(seq)):
        o = (np.zeros(6000, np.uint32), np.zeros(6000, np.float32))
        o1 = (np.zeros(6000, np.uint32), np.zeros(6000, np.float32))
        tk = [srv.submit(srv.ray_request(0, 0, rays, *o)), srv.submit(srv.ray_request(0, 1, rays, *o1))]
        if k + 1 < len(seq):
            tk.append(srv.submit(srv.update_request(0, seq[k + 1])))
        assert all(srv.wait(t) == 0 for t in tk)
        outs.append((k, o, o1))
    ref_other, ref_other_t = _oracle(other, rays, 0)
    for k, o, o1 in outs:
        ref, ref_t = _oracle(seq[k], rays, 0)
        assert np.array_equal(o[0], ref), k
        assert np.array_equal(o[1].view(np.uint32), ref_t.view(np.uint32)), k
        assert np.array_equal(o1[0], ref_other), k
        assert np.array_equal(o1[1].view(np.uint32), ref_other_t.view(np.uint32)), k
    assert srv.stats()["updates"] == len(seq) - 1
    srv.close()


def test_admission_by_memory_budget(gpu):
    import shinobi_b200 as shn
    ctx = shn.Context(0, hbm_budget_bytes=96 << 20)
    srv = shn.Server(ctx=ctx, num_slots=2, max_batch_rays=1 << 16, max_requests_per_launch=64)
    small = scenes.uniform_soup(2000, seed=3)
    srv.load_scene(0, small)
    big = scenes.uniform_soup(1 << 20, seed=4)            # needs far more than the budget
    res = srv.wait(srv.submit(srv.update_request(0, big)))
    assert res == 5                                       # SHN_ERR_BUDGET, old scene kept
    rays = _rays8(4000, 11, 1e30)
    out = (np.zeros(4000, np.uint32), np.zeros(4000, np.float32))
    assert srv.wait(srv.submit(srv.ray_request(0, 0, rays, *out))) == 0
    ref, _ = _oracle(small, rays, 0)
    assert np.array_equal(out[0], ref)
    used, budget = ctx.memory()
    assert used <= budget
    srv.close()
    ctx.close()


def test_rejects_bad_requests(gpu):
    import shinobi_b200 as shn
    srv = shn.Server(num_slots=2, max_batch_rays=1024)
    srv.load_scene(0, scenes.uniform_soup(100, seed=5))
    with pytest.raises(shn.ShinobiError):
        srv.submit(srv.ray_request(0, 0, _rays8(2048, 1, 1e30)))   # above max_batch_rays
    assert srv.wait(srv.submit(srv.ray_request(0, 1, _rays8(10, 1, 1e30)))) == 1   # empty slot: invalid
    srv.close()
