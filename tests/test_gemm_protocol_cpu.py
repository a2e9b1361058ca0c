"""The barrier protocol of the complex GEMM (csrc/gemm_cplx.cu, one-CTA and CTA-pair kernels), restated on the CPU as
a model: mbarriers with a phase count, the producer (waits empty[s] with parity (n & 1) ^ 1 for its n-th use of
stage s, then fills it), the MMA issuer (per item: waits tempty[b] with parity (u & 1) ^ 1, u = item / 2; per K chunk
waits full[s] with parity (f / S) & 1, consumes it and commits empty[s]; commits tfull[b] after the item) and the
epilogue (waits tfull[b] with parity u & 1, reads the accumulator, arrives on tempty[b]). Run under random
interleavings, the model must finish every item and never fill a stage that is still unconsumed, nor start an item
in an accumulator buffer the epilogue has not released."""
import itertools
import random


class Bar:
    """An mbarrier with `count` arrivals per phase; try_wait(parity) is true once the phase with that parity has
    completed (phase k completes when its arrivals reach count; parity of phase k is k & 1)."""

    def __init__(self, count):
        self.count, self.arrived, self.completed = count, 0, 0     # completed phases

    def arrive(self, n=1):
        self.arrived += n
        while self.arrived >= self.count:
            self.arrived -= self.count
            self.completed += 1

    def try_wait(self, parity):
        # the current (incomplete) phase has index `completed`; waiting on parity p succeeds when the most recent
        # completed phase has parity p, i.e. the phase being waited for is done
        return self.completed > 0 and ((self.completed - 1) & 1) == parity or \
            (self.completed == 0 and parity == 1)


def run(S, nkc, ntl, seed):
    rng = random.Random(seed)
    full = [Bar(1) for _ in range(S)]
    empty = [Bar(1) for _ in range(S)]
    tfull = [Bar(1) for _ in range(2)]
    tempty = [Bar(1) for _ in range(2)]
    nfill = ntl * nkc
    stage = [None] * S            # fill index held by each stage, None once consumed
    acc = [None] * 2              # item held by each accumulator buffer, None once released
    state = dict(p=0, m_item=0, m_kc=0, m_started=False, e=0)

    def producer():
        f = state['p']
        if f >= nfill:
            return False
        s, n = f % S, f // S
        if not empty[s].try_wait((n & 1) ^ 1):
            return False
        assert stage[s] is None, 'stage %d refilled before it was consumed' % s
        stage[s] = f
        full[s].arrive()
        state['p'] += 1
        return True

    def mma():
        i = state['m_item']
        if i >= ntl:
            return False
        b, u = i & 1, i >> 1
        if not state['m_started']:
            if not tempty[b].try_wait((u & 1) ^ 1):
                return False
            assert acc[b] is None, 'accumulator %d reused before the epilogue released it' % b
            acc[b] = i
            state['m_started'] = True
            return True
        kc = state['m_kc']
        f = i * nkc + kc
        s = f % S
        if not full[s].try_wait((f // S) & 1):
            return False
        assert stage[s] == f
        stage[s] = None
        empty[s].arrive()                       # commit after the MMAs of this chunk
        state['m_kc'] += 1
        if state['m_kc'] == nkc:
            tfull[b].arrive()                   # commit after the item
            state['m_kc'] = 0
            state['m_item'] += 1
            state['m_started'] = False
        return True

    def epilogue():
        i = state['e']
        if i >= ntl:
            return False
        b, u = i & 1, i >> 1
        if not tfull[b].try_wait(u & 1):
            return False
        assert acc[b] == i
        acc[b] = None
        tempty[b].arrive()
        state['e'] += 1
        return True

    actors = [producer, mma, epilogue]
    steps = 0
    while state['e'] < ntl:
        order = actors[:]
        rng.shuffle(order)
        if not any(a() for a in order):
            raise AssertionError('deadlock at S=%d nkc=%d ntl=%d: %s' % (S, nkc, ntl, state))
        steps += 1
        assert steps < 100000
    assert state['p'] == nfill and state['m_item'] == ntl


def test_gemm_barrier_protocol_completes_under_any_interleaving():
    for S, nkc, ntl in itertools.product([2, 3, 4, 6, 8], [1, 2, 3, 4], [1, 2, 3, 7, 97]):
        for seed in range(5):
            run(S, nkc, ntl, seed)
