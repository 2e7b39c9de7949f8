"""The slot-serving loop: continuous batching into fused launches.

Each slot's LLRs must be bit-identical to the same slot equalized alone by a
single fused launch, whatever else shares its batch; admission holds requests
that do not fit the memory budget until completions free it; a bounded wait
on a paused server returns a timeout status (host-side failure injection, no
GPU fault); SRS updates rewrite the resident channel before later slots."""
from __future__ import annotations

import time

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu

TIMEOUT = 1006


def _alone(aeq, c, H, Y, cuda, plain=False):
    llr = torch.empty(c.llr_numel, dtype=torch.float32, device=cuda)
    d = aeq.cell_desc(H, Y, llr, c.sigma2, c.nPRB, c.nAnt, c.nLayers, c.nSym, c.nPamBits)
    if plain:
        ws = torch.empty(aeq.pusch_eq_plain_workspace([d]), dtype=torch.uint8, device=cuda)
        aeq.pusch_eq_plain([d], ws)
    else:
        aeq.pusch_eq_fused([d])
    torch.cuda.synchronize()
    return llr.cpu().numpy()


def _cells(wl, n, seed):
    shapes = wl.multicell_shapes(n, seed=seed)
    return [wl.make_cell(min(p, 51), a, l, 11, q, snr, "iid", seed=seed + 7 * i)
            for i, (p, a, l, q, snr) in enumerate(shapes)]


@pytest.mark.parametrize("mode", ["fused", "plain"])
def test_server_results_same_alone_and_in_mix(aeq, wl, cuda, mode):
    cells = _cells(wl, 6, 101)
    slots = 3
    with aeq.Server(streams=3, mode=aeq.SERVER_PLAIN if mode == "plain" else aeq.SERVER_FUSED) as srv:
        ids, outs, Ys = [], [], []
        cid = []
        for c in cells:
            k = srv.add_cell(c.nPRB, c.nAnt, c.nLayers, c.nSym, c.nPamBits, c.sigma2)
            srv.set_channel(k, c.H.to(cuda), c.sigma2)
            cid.append(k)
        gens = [[wl.make_cell(c.nPRB, c.nAnt, c.nLayers, c.nSym, 4 ** c.nPamBits, c.snr_db, seed=900 + 31 * i + s)
                 for s in range(slots)] for i, c in enumerate(cells)]
        for s in range(slots):                       # interleave the cells' slots
            for i, c in enumerate(cells):
                Y = gens[i][s].Y.to(cuda)
                out = torch.full((c.llr_numel,), float("nan"), dtype=torch.float32, device=cuda)
                ids.append(srv.submit(cid[i], Y, out))
                outs.append((i, s, out))
                Ys.append(Y)
        srv.drain()
        done = srv.poll()
        assert len(done) == len(ids) and all(st == 0 for _, _, st, _ in done)
        stats = srv.stats()
        assert stats["slots_done"] == len(ids) and stats["p99_us"] >= stats["p50_us"] > 0
    torch.cuda.synchronize()
    for (i, s, out), Y in zip(outs, Ys):
        c = cells[i]
        ref = _alone(aeq, c, c.H.to(cuda), Y, cuda, plain=(mode == "plain"))
        np.testing.assert_array_equal(out.cpu().numpy(), ref)


def test_server_budget_admission_serializes(aeq, wl, cuda):
    c = wl.make_cell(24, 32, 4, 11, 16, 20.0, seed=111)
    h_bytes = 8 * c.nSC * c.nAnt * c.nLayers
    req_bytes = 8 * c.nSC * c.nSym * c.nAnt + 4 * c.llr_numel
    with aeq.Server(memory_budget_bytes=h_bytes + req_bytes, streams=3) as srv:
        k = srv.add_cell(c.nPRB, c.nAnt, c.nLayers, c.nSym, c.nPamBits, c.sigma2)
        srv.set_channel(k, c.H.to(cuda), c.sigma2)
        Y = c.Y.to(cuda)
        outs = [torch.empty(c.llr_numel, dtype=torch.float32, device=cuda) for _ in range(8)]
        for o in outs:
            srv.submit(k, Y, o)
        srv.drain()
        st = srv.stats()
        assert st["slots_done"] == 8
        assert st["mean_batch"] == 1.0                 # one admitted request at a time
        assert st["budget_used_bytes"] == h_bytes       # every request released its share
    ref = _alone(aeq, c, c.H.to(cuda), Y, cuda)
    for o in outs:
        np.testing.assert_array_equal(o.cpu().numpy(), ref)


def test_server_rejects_cell_beyond_budget(aeq, cuda):
    with aeq.Server(memory_budget_bytes=1 << 20, streams=1) as srv:
        with pytest.raises(aeq.AerialError):
            srv.add_cell(132, 64, 8, 11, 4, 0.01)     # 6.5 MB of channel alone


def test_server_bounded_wait_times_out_while_paused(aeq, wl, cuda):
    c = wl.make_cell(4, 16, 2, 11, 4, 15.0, seed=121)
    with aeq.Server(streams=1, start_paused=True) as srv:
        k = srv.add_cell(c.nPRB, c.nAnt, c.nLayers, c.nSym, c.nPamBits, c.sigma2)
        srv.set_channel(k, c.H.to(cuda), c.sigma2)
        out = torch.empty(c.llr_numel, dtype=torch.float32, device=cuda)
        rid = srv.submit(k, c.Y.to(cuda), out)
        t0 = time.monotonic()
        assert srv.wait(rid, timeout_ms=50) == TIMEOUT
        assert time.monotonic() - t0 < 5.0
        assert srv.stats()["pending"] == 1
        srv.pause(False)
        assert srv.wait(rid, timeout_ms=10000) == 0
        assert srv.wait(10 ** 9, timeout_ms=10) == 1007   # unknown request


def test_server_srs_update_rewrites_resident_channel(aeq, orc, wl, cuda):
    K, F = 12, 12
    c = wl.make_cell(2, 32, 4, 11, 16, 20.0, seed=131)
    nBlk = c.nSC // K
    s, w, f = orc.ref_srs_inputs(5, nBlk * c.nAnt * K, K * K, c.nLayers * F)
    dS = torch.from_numpy(s.view(np.int16)).to(cuda)
    dW = torch.from_numpy(w.view(np.int16)).to(cuda)
    dF = torch.from_numpy(f.view(np.int16)).to(cuda)
    Hsrs = torch.empty(c.nSC, c.nAnt, c.nLayers, dtype=torch.complex64, device=cuda)
    aeq.srs_to_channel(Hsrs, dS, dW, dF, c.nAnt, nBlk, K, c.nLayers, F)
    Y = c.Y.to(cuda)
    with aeq.Server(streams=2) as srv:
        k = srv.add_cell(c.nPRB, c.nAnt, c.nLayers, c.nSym, c.nPamBits, c.sigma2)
        srv.set_channel(k, c.H.to(cuda), c.sigma2)
        before = torch.empty(c.llr_numel, dtype=torch.float32, device=cuda)
        after = torch.empty(c.llr_numel, dtype=torch.float32, device=cuda)
        srv.submit(k, Y, before)
        srv.srs_update(k, dS, dW, dF, K, F)
        srv.submit(k, Y, after)
        srv.drain()
        assert srv.stats()["srs_updates"] == 1
    np.testing.assert_array_equal(before.cpu().numpy(), _alone(aeq, c, c.H.to(cuda), Y, cuda))
    np.testing.assert_array_equal(after.cpu().numpy(), _alone(aeq, c, Hsrs, Y, cuda))


def test_server_srs_update_averages_four_symbols(aeq, orc, wl, cuda):
    """An SRS update over 4 SRS symbols (the serving configuration's) leaves the
    resident channel equal to srs_to_channel_avg of those symbols: the slot
    queued after it equalizes bit for bit like a launch on that channel."""
    K, F, S = 12, 4, 4
    c = wl.make_cell(4, 64, 4, 11, 64, 25.0, seed=133)
    nBlk = c.nSC // K
    syms = [orc.ref_srs_inputs(70 + q, nBlk * c.nAnt * K, K * K, c.nLayers * F) for q in range(S)]
    dS = torch.from_numpy(np.concatenate([x[0] for x in syms]).view(np.int16)).to(cuda)
    dW = torch.from_numpy(syms[0][1].view(np.int16)).to(cuda)
    dF = torch.from_numpy(syms[0][2].view(np.int16)).to(cuda)
    Havg = torch.empty(c.nSC, c.nAnt, c.nLayers, dtype=torch.complex64, device=cuda)
    aeq.srs_to_channel_avg(Havg, dS, S, dW, dF, c.nAnt, nBlk, K, c.nLayers, F)
    Y = c.Y.to(cuda)
    with aeq.Server(streams=2) as srv:
        k = srv.add_cell(c.nPRB, c.nAnt, c.nLayers, c.nSym, c.nPamBits, c.sigma2)
        srv.set_channel(k, c.H.to(cuda), c.sigma2)
        after = torch.empty(c.llr_numel, dtype=torch.float32, device=cuda)
        srv.srs_update(k, dS, dW, dF, K, F, n_symbols=S)
        srv.submit(k, Y, after)
        srv.drain()
        assert srv.stats()["srs_updates"] == 1
        with pytest.raises(aeq.AerialError):
            srv.srs_update(k, dS, dW, dF, K, F, n_symbols=3)
    np.testing.assert_array_equal(after.cpu().numpy(), _alone(aeq, c, Havg, Y, cuda))


def test_server_deadline_misses_counted_for_late_producer(aeq, wl, cuda):
    """Fault injected on the host: a producer that hands slots over late (arrival stamped 200 ms before the
    submit, on the same steady clock) makes every such slot miss a 20 ms deadline, and the statistics count
    them; slots handed over on time do not miss.  Malformed submissions return codes and queue nothing."""
    c = wl.make_cell(4, 16, 2, 11, 4, 15.0, seed=131)
    with aeq.Server(streams=1, deadline_us=20000.0) as srv:
        k = srv.add_cell(c.nPRB, c.nAnt, c.nLayers, c.nSym, c.nPamBits, c.sigma2)
        srv.set_channel(k, c.H.to(cuda), c.sigma2)
        Y = c.Y.to(cuda)
        outs = [torch.empty(c.llr_numel, dtype=torch.float32, device=cuda) for _ in range(8)]
        for o in outs[:4]:
            srv.submit(k, Y, o, arrival_ns=time.monotonic_ns() - 200_000_000)
        srv.drain()
        st = srv.stats()
        assert st["slots_done"] == 4 and st["deadline_misses"] == 4
        srv.reset_stats()
        for o in outs[4:]:
            srv.submit(k, Y, o)
        srv.drain()
        st = srv.stats()
        assert st["slots_done"] == 4 and st["deadline_misses"] == 0
        assert srv.submit_status(k + 100, Y, outs[0]) == 1007     # unknown cell
        assert srv.submit_status(k, None, outs[0]) == 1001        # null received samples
        assert srv.submit_status(k, Y, None) == 1001              # null LLR buffer
        assert srv.stats()["pending"] == 0
        torch.cuda.synchronize()
        for o in outs[1:]:
            assert torch.equal(o, outs[0])                        # same slot, same LLRs, late or not


@pytest.mark.parametrize("mode,nth", [("fused", 1), ("plain", 1), ("plain", 3)])
def test_server_allocation_failure_leaves_server_usable(aeq, wl, cuda, mode, nth):
    """A device allocation that fails inside add_cell (injected on the host:
    the runtime is not called) leaves the server as it was: no cell added, the
    budget unchanged, and the cell already there serves bit-identical results.
    nth = 1 fails the channel's allocation; in the plain mode with two streams
    nth = 3 fails the second workspace of the regrowth, after the channel and
    the first workspace were allocated.  The same cell then adds cleanly."""
    plain = mode == "plain"
    small = wl.make_cell(4, 16, 2, 11, 4, 15.0, seed=131)
    big = wl.make_cell(24, 32, 4, 11, 16, 20.0, seed=132)
    with aeq.Server(streams=2, mode=aeq.SERVER_PLAIN if plain else aeq.SERVER_FUSED) as srv:
        Hs = small.H.to(cuda)
        k0 = srv.add_cell(small.nPRB, small.nAnt, small.nLayers, small.nSym, small.nPamBits, small.sigma2)
        srv.set_channel(k0, Hs, small.sigma2)
        used = srv.stats()["budget_used_bytes"]
        srv.inject_alloc_failure(nth)
        with pytest.raises(aeq.AerialError) as err:
            srv.add_cell(big.nPRB, big.nAnt, big.nLayers, big.nSym, big.nPamBits, big.sigma2)
        assert err.value.status == 2                                   # cudaErrorMemoryAllocation
        assert srv.stats()["budget_used_bytes"] == used
        Ys = small.Y.to(cuda)
        out = torch.full((small.llr_numel,), float("nan"), dtype=torch.float32, device=cuda)
        assert srv.wait(srv.submit(k0, Ys, out)) == 0
        np.testing.assert_array_equal(out.cpu().numpy(), _alone(aeq, small, Hs, Ys, cuda, plain))
        k1 = srv.add_cell(big.nPRB, big.nAnt, big.nLayers, big.nSym, big.nPamBits, big.sigma2)
        assert k1 == k0 + 1
        Hb, Yb = big.H.to(cuda), big.Y.to(cuda)
        srv.set_channel(k1, Hb, big.sigma2)
        outs = [torch.full((c.llr_numel,), float("nan"), dtype=torch.float32, device=cuda) for c in (small, big)]
        ids = [srv.submit(k0, Ys, outs[0]), srv.submit(k1, Yb, outs[1])]
        assert all(srv.wait(i) == 0 for i in ids)
    np.testing.assert_array_equal(outs[0].cpu().numpy(), _alone(aeq, small, Hs, Ys, cuda, plain))
    np.testing.assert_array_equal(outs[1].cpu().numpy(), _alone(aeq, big, Hb, Yb, cuda, plain))


def test_server_plain_workspace_regrowth_while_slots_in_flight(aeq, wl, cuda):
    """In the plain mode a larger cell regrows every stream's workspace.  Added
    while slots of a smaller cell are queued and running, it waits until no
    batch holds the old workspaces, so every slot's LLRs stay bit-identical."""
    small = wl.make_cell(24, 32, 2, 11, 16, 20.0, seed=141)
    big = wl.make_cell(51, 64, 8, 11, 64, 25.0, seed=142)
    with aeq.Server(streams=3, mode=aeq.SERVER_PLAIN) as srv:
        Hs, Ys = small.H.to(cuda), small.Y.to(cuda)
        k0 = srv.add_cell(small.nPRB, small.nAnt, small.nLayers, small.nSym, small.nPamBits, small.sigma2)
        srv.set_channel(k0, Hs, small.sigma2)
        outs = [torch.full((small.llr_numel,), float("nan"), dtype=torch.float32, device=cuda) for _ in range(24)]
        ids = [srv.submit(k0, Ys, o) for o in outs]
        k1 = srv.add_cell(big.nPRB, big.nAnt, big.nLayers, big.nSym, big.nPamBits, big.sigma2)
        Hb, Yb = big.H.to(cuda), big.Y.to(cuda)
        srv.set_channel(k1, Hb, big.sigma2)
        ob = torch.full((big.llr_numel,), float("nan"), dtype=torch.float32, device=cuda)
        ids.append(srv.submit(k1, Yb, ob))
        outs += [torch.full_like(outs[0], float("nan")) for _ in range(4)]
        ids += [srv.submit(k0, Ys, o) for o in outs[-4:]]
        assert all(srv.wait(i) == 0 for i in ids)
    ref = _alone(aeq, small, Hs, Ys, cuda, plain=True)
    for o in outs:
        np.testing.assert_array_equal(o.cpu().numpy(), ref)
    np.testing.assert_array_equal(ob.cpu().numpy(), _alone(aeq, big, Hb, Yb, cuda, plain=True))


def test_real_allocation_failure_does_not_leak_into_the_next_launch(aeq, wl, cuda):
    """A real cudaMalloc failure (a 206 GB channel at the largest cell the
    envelope allows: the runtime refuses it and touches no memory) is returned
    by add_cell and cleared from this thread's last-error state, so the next
    launch on the thread reports its own success rather than the old
    failure."""
    with aeq.Server(memory_budget_bytes=1 << 50, streams=1) as srv:
        with pytest.raises(aeq.AerialError) as err:
            srv.add_cell(aeq.MAX_PRB + 1, 16, 2, 11, 4, 0.01)
        assert err.value.status == 1001                       # beyond the envelope: checked on the host
        with pytest.raises(aeq.AerialError) as err:
            srv.add_cell(aeq.MAX_PRB, 256, 16, 14, 4, 0.01)  # 8 B x 6.3 M subcarriers x 256 x 16
        assert err.value.status == 2                          # cudaErrorMemoryAllocation
        assert srv.stats()["budget_used_bytes"] == 0
    c = wl.make_cell(4, 16, 2, 11, 4, 15.0, seed=151)
    llr = _alone(aeq, c, c.H.to(cuda), c.Y.to(cuda), cuda)    # raises if its launch check saw the old error
    assert np.isfinite(llr).all()
