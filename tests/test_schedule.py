"""The adjoint-pass launch programs, checked on the host.

The engine keeps only the forward checkpoint pairs and rebuilds the other forward
fields segment by segment (checkpoint.c:130-265, propagation.c:641-673).  With overlap,
the rebuild of segment k-1 runs in the same launches as the adjoint steps of segment
k.  The two-step kernel's program (overlap 2) advances up to two replay steps and two adjoint
steps per launch.  This test replays a program symbolically: every frame buffer holds the
time index of the field it contains, items of one launch read the state before the launch
and write after it, every read must find the field its step needs, and no launch writes a
buffer that it also reads (the blocks of a launch read halos of each other's inputs).  The
buffer mapping below restates the device's (fwi_kernels.cuh: stored_slot, seg_idx, rep_idx,
adj_idx; fields that are not kept rotate through four frames).
"""
import ctypes as C

import numpy as np
import pytest

from fwiedu import engine as E

K_NONE, K_REP, K_ADJ = 0, 3, 4
DEPTH2 = 0x100
NROT = 4


def program(nt, overlap):
    L = E.lib()
    n = L.fwi_adjoint_program(nt, overlap, None, 0)
    buf = (C.c_int * (4 * n))()
    assert L.fwi_adjoint_program(nt, overlap, buf, n) == n
    return np.frombuffer(buf, np.int32).reshape(n, 4)


class Buffers:
    def __init__(self, nt):
        self.nt = nt
        self.d = E.lib().fwi_checkpoint_interval(nt)
        self.S5 = self.d // 5 + 2

    def slot(self, t):
        d, nt = self.d, self.nt
        if t == -1:
            return 0
        if t < 0 or t >= nt:
            return -1
        if t % d == 0:
            return 2 * (t // d) + 1
        if (t + 1) % d == 0 and t + 1 < nt:
            return 2 * ((t + 1) // d)
        return -1

    def seg(self, t):
        k = t // self.d
        c = k * self.d
        j = t // 5 - (c + 5) // 5
        assert 0 <= j < self.S5
        return ("seg", (k & 1) * self.S5 + j)

    def rep(self, t):
        s = self.slot(t)
        if s >= 0:
            return ("ck", s)
        if t % 5 == 0:
            return self.seg(t)
        return ("rscr", t % NROT)

    def adj(self, t):
        return ("adj", (t + NROT) % NROT)

    def img(self, t):
        s = self.slot(t)
        return ("ck", s) if s >= 0 else self.seg(t)


def simulate(nt, overlap):
    B = Buffers(nt)
    state = {}
    for t in range(-1, nt):  # the forward pass leaves the checkpoint pairs
        s = B.slot(t)
        if s >= 0:
            state[("ck", s)] = t
    state[B.adj(nt)] = nt          # the adjoint pass starts from A(nt) = 0 and A(nt - 1)
    state[B.adj(nt - 1)] = nt - 1
    adj_seen = []
    rep_seen = []
    for launch in program(nt, overlap):
        reads, writes = [], []
        for kw, step in ((launch[0], launch[1]), (launch[2], launch[3])):
            kind, steps = kw & 0xFF, (2 if kw & DEPTH2 else 1)
            if kind == K_REP:
                reads += [(B.rep(step), step), (B.rep(step - 1), step - 1)]
                for j in range(steps):
                    writes.append((B.rep(step + 1 + j), step + 1 + j))
                    rep_seen.append(step + j)
            elif kind == K_ADJ:
                reads += [(B.adj(step), step), (B.adj(step + 1), step + 1)]
                for j in range(steps):
                    t = step - j
                    if t % 5 == 0:
                        reads.append((B.img(t), t))
                    writes.append((B.adj(t - 1), t - 1))
                    adj_seen.append(t)
            else:
                assert kind == K_NONE
        for buf, want in reads:
            assert state.get(buf) == want, f"nt={nt}: {buf} holds {state.get(buf)}, step needs {want}"
        wb = [w[0] for w in writes]
        assert len(wb) == len(set(wb))
        assert not set(wb) & {r[0] for r in reads}, "a launch writes a buffer it also reads"
        for buf, val in writes:
            state[buf] = val
    return adj_seen, rep_seen, B


@pytest.mark.parametrize("nt", [1, 2, 3, 4, 7, 10, 37, 100, 200, 201, 299, 300, 451, 1000, 4001])
@pytest.mark.parametrize("overlap", [0, 1, 2])
def test_program_feeds_every_imaging_step(nt, overlap):
    adj, rep, B = simulate(nt, overlap)
    assert adj == list(range(nt - 1, -1, -1))
    # each non-stored step is rebuilt exactly once
    nonstored = [t for t in range(nt) if B.slot(t) < 0]
    assert sorted(s + 1 for s in rep) == nonstored


def test_overlap_removes_most_replay_launches():
    nt = 4001
    plain = len(program(nt, 0))
    over = len(program(nt, 1))
    assert plain == nt + (nt - 89)  # the reference's 3912 replay steps, one launch each
    assert over < nt + 2 * 89  # replay hidden behind the adjoint steps except the last segment


def test_two_step_program_halves_the_launches():
    nt = 4001
    one = len(program(nt, 1))
    two = len(program(nt, 2))
    assert two < 0.55 * one
