"""Edge cases of the device decoders against the oracle, both engines:
a container taller than the top-z index covers (binary-search path), items
that never fit, types with zero quantity or no allowed orientation, a single
item, and one long run of identical items (the incremental path throughout).
Every restart's JSON (time_s removed) must be identical."""
import random

import pytest

import oracle_py as O
import plpb200 as P
from plpb200 import synth

pytestmark = pytest.mark.gpu


def thpack(L, W, H, types):
    lines = ["1", "1 1", f"{L} {W} {H}", str(len(types))]
    for i, (l, lf, w, wf, h, hf, q) in enumerate(types, 1):
        lines.append(f"{i} {l} {lf} {w} {wf} {h} {hf} {q}")
    return "\n".join(lines) + "\n"


def tall():
    rng = random.Random(4)
    return thpack(50, 40, 5000, [(rng.randint(8, 25), 1, rng.randint(8, 20), 1, rng.randint(20, 90), 1,
                                  rng.randint(20, 60)) for _ in range(4)])


CASES = {
    "tall_container_no_z_index": tall(),
    "nothing_fits": thpack(100, 100, 100, [(150, 1, 20, 1, 20, 0, 5), (120, 0, 130, 0, 140, 1, 3)]),
    "zero_qty_and_no_orientation": thpack(200, 150, 120, [(40, 1, 30, 1, 20, 1, 0), (50, 0, 40, 0, 30, 0, 4),
                                                          (35, 1, 25, 0, 15, 1, 9), (60, 1, 45, 1, 30, 1, 5)]),
    "single_item": thpack(300, 200, 100, [(80, 1, 60, 1, 40, 1, 1)]),
    "one_long_run": thpack(400, 250, 200, [(37, 1, 29, 1, 23, 1, 180)]),
    # footprints of 300 x 300 >= 65536: contact areas stay 32-bit
    "large_footprints_32bit_areas": thpack(1000, 1000, 100, [(300, 1, 300, 1, 40, 1, 9), (250, 1, 180, 1, 30, 1, 14),
                                                             (90, 1, 70, 1, 20, 1, 30)]),
}


@pytest.fixture(scope="module")
def handle():
    with P.Handle() as h:
        yield h


@pytest.mark.parametrize("name", sorted(CASES))
@pytest.mark.parametrize("eps", [0.0, 0.3])
def test_decoder_edge_cases_match_oracle(handle, name, eps):
    text = CASES[name]
    r = handle.solve([P.Instance.parse(text)], P.make_opts(seed=9, restarts=12, eps=eps, passes=2))[0]
    oi = O.OInstance(text)
    for k in range(12):
        js, _, _ = O.run(oi, seed=9 + k, passes=2, eps=eps)
        assert O.strip_time(r.json(k)) == O.strip_time(js), (name, k)


@pytest.mark.parametrize("name", sorted(CASES))
@pytest.mark.parametrize("pick", ["first", "contact"])
def test_block_engine_edge_cases_match_oracle(handle, name, pick):
    text = CASES[name]
    r = handle.solve([P.Instance.parse(text)],
                     P.make_opts(seed=9, restarts=12, eps=0.4, passes=2, engine="block", pick=pick))[0]
    oi = O.OInstance(text)
    for k in range(12):
        js = O.run_block(oi, seed=9 + k, passes=2, eps=0.4, pick=pick)
        assert O.strip_time(r.json(k)) == O.strip_time(js), (name, k)


@pytest.mark.parametrize("G", [2, 4])
def test_bounded_barrier_wait_gives_up_with_a_device_error(G):
    """The multi-warp decoder's barrier waits are bounded. With the test hook
    one warp of every decoder leaves out its first arrive, so each decoder's
    first wait runs out after 256 tries (about 3 ms at most); the launch ends
    with the barrier error, the solve returns PLP_E_DEVICE instead of hanging,
    and the same handle then solves correctly once the hook is cleared."""
    text = synth.multi_restart(2).to_thpack()
    inst = P.Instance.parse(text)
    with P.Handle() as h:
        h.set_tile(P=128, C=384, G=G, D=1, M=1)
        h.debug_sync_bound(wait_limit=256, skip_warp=G - 1)
        with pytest.raises(P.PlpError) as e:
            h.solve([inst], P.make_opts(seed=0, restarts=8))
        assert e.value.status == P.E_DEVICE
        assert "barrier" in str(e.value)
        h.debug_sync_bound(0, -1)
        res = h.solve([inst], P.make_opts(seed=0, restarts=8))[0]
    oi = O.OInstance(text)
    for k in range(8):
        js, _, _ = O.run(oi, seed=k)
        assert O.strip_time(res.json(k)) == O.strip_time(js)
