"""Request server (continuous batching): a request gives the same result alone and in a
mix with other lattices and sector sizes, arriving while others run; results match the
plain driver; FP32 storage with FP64 refinement stays within 1e-8 of FP64; admission
respects the HBM budget."""
import pytest

import hphi_b200
from hphi_b200 import expert

pytestmark = pytest.mark.gpu


def _kw():
    return dict(lanczos_max=400, lanczos_eps=12, lanczos_target=1)


REQUESTS = [
    ("heis10", lambda: expert.heisenberg(10, expert.chain_bonds(10), 1.0, **_kw())),
    ("heis14", lambda: expert.heisenberg(14, expert.chain_bonds(14), 1.0, **_kw())),
    ("hub6_u4", lambda: expert.hubbard(6, expert.chain_bonds(6), 1.0, 4.0, 3, 3, **_kw())),
    ("hub8_u8", lambda: expert.hubbard(8, expert.chain_bonds(8), 1.0, 8.0, 4, 4, **_kw())),
    ("kh_gc8", lambda: expert.kitaev_heisenberg(2, 2, -1.0, 0.15, initial_vec_type=0, **_kw())),
    ("j1j2_12", lambda: expert.j1j2_chain(12, 1.0, 0.3, **_kw())),
]


@pytest.fixture(scope="module")
def inputs(tmp_path_factory):
    return [make().write(str(tmp_path_factory.mktemp(name))) for name, make in REQUESTS]


def _drain(srv, ids, max_iter=5000):
    got = {}
    for _ in range(max_iter):
        srv.step()
        for rid, d in srv.poll():
            got[rid] = d
        if all(i in got for i in ids):
            return got
    raise AssertionError("server did not finish")


def _serve(inputs, precision=hphi_b200.FP64, staggered=False, **kw):
    with hphi_b200.Server(precision=precision, **kw) as srv:
        ids = []
        half = len(inputs) // 2 if staggered else len(inputs)
        for k, path in enumerate(inputs[:half]):
            ids.append(srv.submit(path, seed=100 + k))
        if staggered:  # the rest arrive while the first ones are on the GPU
            srv.step()
            srv.step()
            for k, path in enumerate(inputs[half:], start=half):
                ids.append(srv.submit(path, seed=100 + k))
        got = _drain(srv, ids)
    return [got[i] for i in ids]


def _alone(inputs, precision=hphi_b200.FP64):
    out = []
    for k, path in enumerate(inputs):
        with hphi_b200.Server(precision=precision) as srv:
            rid = srv.submit(path, seed=100 + k)
            out.append(_drain(srv, [rid])[rid])
    return out


def test_serve_same_result_alone_and_in_mix(inputs):
    alone = _alone(inputs)
    mixed = _serve(inputs, staggered=True)
    for (name, _), a, m in zip(REQUESTS, alone, mixed):
        assert a["status"] == 0 and m["status"] == 0, name
        assert m["energy"] == a["energy"], (name, m["energy"], a["energy"])
        assert m["steps"] == a["steps"], name
        assert m["latency_s"] > 0 and m["wait_s"] >= 0


def test_serve_matches_plain_driver(inputs):
    served = _serve(inputs)
    for k, ((name, _), path, r) in enumerate(zip(REQUESTS, inputs, served)):
        with hphi_b200.Hamiltonian(path) as H:
            e = H.lanczos_steps(min(300, H.dim), seed=100 + k, nev=1)[0]
            assert r["dim"] == H.dim
        assert abs(r["energy"] - e) < 1e-9, (name, r["energy"], e)


def test_serve_fp32_refined_within_1e8(inputs):
    r64 = _serve(inputs)
    r32 = _serve(inputs, precision=hphi_b200.FP32, staggered=True)
    for (name, _), a, b in zip(REQUESTS, r64, r32):
        assert b["status"] == 0, name
        assert abs(b["energy"] - a["energy"]) < 1e-8, (name, b["energy"], a["energy"])
        assert b["residual"] < 1e-3, name


def test_serve_budget_admission_and_oversized_request(inputs, tmp_path):
    # a budget that holds about one request at a time still serves everything, identically
    tight = _serve(inputs, hbm_budget=3 << 19)
    free = _serve(inputs)
    for (name, _), a, b in zip(REQUESTS, tight, free):
        assert a["energy"] == b["energy"], name
    big = expert.heisenberg(20, expert.chain_bonds(20), 1.0, **_kw()).write(str(tmp_path))
    with hphi_b200.Server(hbm_budget=1 << 20) as srv:
        rid = srv.submit(big)
        got = _drain(srv, [rid])[rid]
    assert got["status"] == -1 and "budget" in got["error"]
