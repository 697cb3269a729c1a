"""The P2P halo protocol of fv_group_run (finite-volume-2d-cpp_b200/csrc/
fv_group.cu: group_step, k_p2p_push, k_p2p_wait; and the same schedule
inside the fused stage launch, fv_fused.cuh fused_tile<..., REMOTE>), checked
as a model under random interleavings of the processes.

Each simulated process owns one part and runs the step schedule of
group_step with the P2P transport:
- wait for every sender's epoch step*S + 0, then the dt kernel reads the
  halo of the step's input buffer;
- the dt all-gather (no process passes before every process has arrived);
- per stage k: (k > 0) wait for step*S + k; the band tiles read the halo of
  the stage's input buffer; the push stores this part's states into every
  reader's buffer of stage k's output role and releases step*S + k + 1;
- the residual all-gather, the step end.
Buffer roles are those of step_stage: tmp[k % 2] for the inner stages,
sbase[b] for the last stage, sbase[1 - b] for RK1, b alternating between
RK1 steps.

Every halo cell carries the (step, stage) of the push that wrote it.  Each
read must see exactly the version its stage needs: a read before the push
arrived (a wait too short) or after a later push overwrote it (a push too
early into a buffer the reader still reads) fails the test.
"""
import random

import pytest


def role_of(S, k, b):
    return 2 + (1 - b) if S == 1 else (2 + b if k == S - 1 else k % 2)


def input_role(S, k, b):
    return 2 + b if k == 0 else role_of(S, k - 1, b)


def run_model(n_proc, S, steps, seed):
    rng = random.Random(seed)
    P = n_proc
    # halo[r][role][s]: version (step, stage) of sender s's states in reader r's buffer
    halo = [[[None] * P for _ in range(4)] for _ in range(P)]
    for r in range(P):
        for s in range(P):
            halo[r][2][s] = ("initial",)      # sbase[0] holds the initial state
    flags = [[0] * P for _ in range(P)]       # flags[r][s]: last epoch s released to r
    barrier = {}                              # name -> set of arrived processes
    log = []

    def expected(S, n, k, b):
        """The version stage k of step n reads in its input buffer."""
        if k > 0:
            return (n, k - 1)
        if n == 0:
            return ("initial",)
        return (n - 1, S - 1)

    def proc(p):
        for n in range(steps):
            b = (n % 2) if S == 1 else 0
            # wait for the previous step's last stage
            need = n * S
            while any(flags[p][s] < need for s in range(P) if s != p):
                yield "wait"
            # dt kernel reads the input halo
            for s in range(P):
                if s != p:
                    got = halo[p][input_role(S, 0, b)][s]
                    assert got == expected(S, n, 0, b), ("dt", p, n, s, got)
            # dt all-gather
            key = ("dt", n)
            barrier.setdefault(key, set()).add(p)
            while len(barrier[key]) < P:
                yield "barrier"
            for k in range(S):
                if k > 0:
                    need = n * S + k
                    while any(flags[p][s] < need for s in range(P) if s != p):
                        yield "wait"
                # band tiles read the stage's input halo
                for s in range(P):
                    if s != p:
                        got = halo[p][input_role(S, k, b)][s]
                        assert got == expected(S, n, k, b), ("band", p, n, k, s, got)
                yield "band"
                # push into every reader's output-role buffer, then release
                for r in range(P):
                    if r != p:
                        halo[r][role_of(S, k, b)][p] = (n, k)
                yield "push"
                for r in range(P):
                    if r != p:
                        flags[r][p] = n * S + k + 1
                log.append((p, n, k))
                yield "interior"
            key = ("R", n)
            barrier.setdefault(key, set()).add(p)
            while len(barrier[key]) < P:
                yield "barrier"

    gens = {p: proc(p) for p in range(P)}
    live = set(gens)
    ticks = 0
    while live:
        p = rng.choice(sorted(live))
        try:
            next(gens[p])
        except StopIteration:
            live.discard(p)
        ticks += 1
        assert ticks < 10 ** 6, "no progress (deadlock)"
    return log


@pytest.mark.parametrize("S", [5, 1, 3])
@pytest.mark.parametrize("n_proc", [2, 3])
def test_p2p_epochs_order_every_halo_read(S, n_proc):
    for seed in range(40):
        log = run_model(n_proc, S, steps=6, seed=seed)
        assert len(log) == n_proc * 6 * S


def test_the_model_catches_a_wait_one_epoch_short():
    """The same model with every wait one epoch short reads stale halos."""
    import test_exchange_protocol as m

    def short_run(seed):
        rng = random.Random(seed)
        P, S, steps = 2, 5, 4
        halo = [[[("initial",)] * P if role == 2 else [None] * P for role in range(4)] for _ in range(P)]
        flags = [[0] * P for _ in range(P)]
        bad = []

        def proc(p):
            for n in range(steps):
                for k in range(S):
                    need = n * S + k - 1          # one short
                    while any(flags[p][s] < need for s in range(P) if s != p):
                        yield
                    want = ("initial",) if (n, k) == (0, 0) else ((n, k - 1) if k > 0 else (n - 1, S - 1))
                    for s in range(P):
                        if s != p and halo[p][m.input_role(S, k, 0)][s] != want:
                            bad.append((p, n, k))
                    yield
                    for r in range(P):
                        if r != p:
                            halo[r][m.role_of(S, k, 0)][p] = (n, k)
                    yield
                    for r in range(P):
                        if r != p:
                            flags[r][p] = n * S + k + 1
                    yield

        gens = [proc(p) for p in range(P)]
        live = set(range(P))
        while live:
            p = rng.choice(sorted(live))
            try:
                next(gens[p])
            except StopIteration:
                live.discard(p)
        return bad

    assert any(short_run(seed) for seed in range(40))
