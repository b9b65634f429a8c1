"""Model check of the cp.async pipelines in bcl_b200/csrc/spmm.cu (no GPU).

The sequences below mirror the issue / commit / wait / build / apply order of
`spmm_rows` (A entries staged kARing = 4 chunks ahead, tables built two
chunks ahead, one commit group per issue) and `spmm_long_row` (A staged six
chunks ahead, B-row slices two chunks ahead, one group per chunk step).  For
every chunk count the model asserts that a chunk is built only after its A
copies have landed, applied only after its B copies have landed and its
table holds it, and that no staging, B or table slot is reused before its
previous chunk was consumed.  A change to either pipeline changes this
sequence too."""
import pytest


class Sim:
    def __init__(self, nch, aslots, bslots, tslots):
        self.nch, self.aslots, self.bslots, self.tslots = nch, aslots, bslots, tslots
        self.groups = []          # committed groups: list of sets of ('A'|'B', chunk)
        self.open = set()         # copies issued since the last commit
        self.landed = set()
        self.aslot = {}           # slot -> chunk staged there
        self.bslot = {}
        self.tab = {}
        self.built = set()
        self.applied = set()

    def issue_a(self, x):
        if x >= self.nch: return
        s = x % self.aslots
        prev = self.aslot.get(s)
        assert prev is None or prev in self.built, f"A slot {s} reused for {x} before chunk {prev} was built"
        self.aslot[s] = x
        self.open.add(('A', x))

    def issue_b(self, x):
        if x >= self.nch: return
        assert self.tab.get(x % self.tslots) == x, f"B copies of {x} without its table"
        s = x % self.bslots
        prev = self.bslot.get(s)
        assert prev is None or prev in self.applied, f"B slot {s} reused for {x} before chunk {prev} was applied"
        self.bslot[s] = x
        self.open.add(('B', x))

    def commit(self):
        self.groups.append(self.open); self.open = set()

    def wait(self, n):
        done = self.groups[:len(self.groups) - n] if n else self.groups
        for g in done: self.landed |= g

    def build(self, x):
        if x >= self.nch: return
        assert ('A', x) in self.landed, f"build {x} before A landed"
        s = x % self.tslots
        prev = self.tab.get(s)
        assert prev is None or prev in self.applied, f"table slot {s} reused for {x} before {prev} applied"
        self.tab[s] = x; self.built.add(x)

    def apply(self, c, need_b):
        assert self.tab.get(c % self.tslots) == c, f"apply {c}: table holds {self.tab.get(c % self.tslots)}"
        if need_b: assert ('B', c) in self.landed, f"apply {c} before B landed"
        self.applied.add(c)


def spmm_rows(nch, P=4):
    s = Sim(nch, P, 1, 3)
    def ia(x): s.issue_a(x); s.commit()   # issue_a commits every call
    for x in range(P): ia(x)
    s.wait(P - 2); s.build(0); s.build(1); ia(P)
    for c in range(nch):
        ia(c + P + 1); s.wait(P - 1); s.build(c + 2); s.apply(c, False)


def spmm_long_row(nch):
    s = Sim(nch, 6, 3, 3)
    s.issue_a(0); s.issue_a(1); s.commit(); s.issue_a(2); s.issue_a(3); s.commit(); s.wait(1)
    s.build(0); s.build(1)
    s.issue_b(0); s.issue_a(4); s.commit(); s.issue_b(1); s.issue_a(5); s.commit(); s.wait(2)
    for c in range(nch):
        s.issue_a(c + 6); s.build(c + 2); s.issue_b(c + 2); s.commit(); s.wait(2); s.apply(c, True)


@pytest.mark.parametrize("nch", list(range(1, 41)))
def test_spmm_rows_pipeline(nch):
    spmm_rows(nch)


@pytest.mark.parametrize("nch", list(range(1, 41)))
def test_spmm_long_row_pipeline(nch):
    spmm_long_row(nch)
