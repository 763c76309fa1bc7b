"""CPU checks of the lag kernel's launch tables and its shared-memory pipeline protocol.

The lag kernel (cuda_multiddm_b200/csrc/lag.cuh) streams the distinct partner frames of a
launch (the "union") through groups of 8 shared-memory slots (8 groups for up to 32
register frames, 16 for 64): one producer lane issues each group's 2-D TMA boxes and arms
the group's *full* barrier; four consumer warps wait once per window on every group it
reaches and arrive on a group's *empty* barrier once no later window reads it. These tests
build the tables with the engine's own C++ builder
(``build_lag_table``, csrc/lag_host.hpp, driven by tests/lag_table_probe.cu) for the
schedules the engine launches — causal windows (unbiased estimator) and the reference's
start|end windows (src/DDM.cu:250-255) — plus random windows with holes, and check

* every window maps union entries back to the ring slots of its positions,
* the TMA runs cover exactly the union entries that hold a frame, inside their group,
* the "full window" flag is right (it selects the kernel's unchecked fast paths),
* the table fits the kernel's shared-memory limit,
* a replay of the barrier protocol (mbarrier phase parity as the hardware defines it) under
  random interleavings of the producer and the four consumer warps, over one element block
  and over several (the persistent grid walks many per CTA, the group counter running on),
  neither deadlocks nor lets a consumer read a slot that holds another group's data.
"""
from __future__ import annotations

import os
import random
import subprocess
import sys
from pathlib import Path

import pytest

from cuda_multiddm_b200.media import log_taus

ROOT = Path(__file__).resolve().parents[1]
CSRC = ROOT / "cuda_multiddm_b200" / "csrc"
PROBE_SRC = ROOT / "tests" / "lag_table_probe.cu"
PROBE = ROOT / "tests" / "_build" / "lag_table_probe"

# constants of csrc/lag.cuh
GROUP, CONSUMERS = 8, 4
FUSE, FULL_FLAG, RUN_FLAG = 4, 1, 2
ACC_SLOTS = 4
LAG_JS = (4, 8, 16, 20, 24, 30, 32, 64)
SMEM_MAX = 220 * 1024
TAB_ENTRIES = 5 + 64


def ring_slots(J: int) -> int:
    return 128 if J > 32 else 64


def slot_bytes(J: int) -> int:
    return 512 if J > 32 else 1024  # a CTA's element block: 64 (two lanes each) or 128 elements


def pick_j(nreg: int) -> int:
    return next(j for j in LAG_JS if j >= nreg)


@pytest.fixture(scope="module")
def probe() -> Path:
    deps = [PROBE_SRC, CSRC / "lag_host.hpp", CSRC / "lag.cuh"]
    if not PROBE.exists() or PROBE.stat().st_mtime < max(p.stat().st_mtime for p in deps):
        PROBE.parent.mkdir(parents=True, exist_ok=True)
        # built under a private name and renamed into place, so parallel test workers never
        # run a half-written binary
        tmp = PROBE.with_name(f"{PROBE.name}.{os.getpid()}")
        subprocess.run(["nvcc", "-std=c++17", "-O1", "-gencode", "arch=compute_100a,code=sm_100a",
                        "-I", str(CSRC), str(PROBE_SRC), "-o", str(tmp)], check=True)
        os.replace(tmp, PROBE)
    return PROBE


def build_tables(probe: Path, cases: list[dict]) -> list[list[int] | str]:
    lines = []
    for c in cases:
        nreg = c["nreg"]
        vals = [nreg, pick_j(nreg), len(c["ent_acc"]), len(c["pos"])]
        vals += c["reg"][:nreg] + c["ent_acc"] + c["ent_w"] + c["pos"]
        lines.append(" ".join(map(str, vals)))
    out = subprocess.run([str(probe)], input="\n".join(lines) + "\n", capture_output=True, text=True,
                         check=True).stdout.splitlines()
    assert len(out) == len(cases)
    return [o if o.startswith("ERR") else [int(v) for v in o.split()] for o in out]


def parse(t: list[int]) -> dict:
    nreg, ntau, nu, ngroups, nruns = t[:5]
    p = TAB_ENTRIES
    d = {"nreg": nreg, "ntau": ntau, "nu": nu, "ngroups": ngroups, "reg": t[5:5 + 64]}
    for name, n in (("ent_acc", ntau), ("ub", ntau), ("full", ntau), ("uslot", nu),
                    ("gptr", ngroups + 1), ("runs", nruns)):
        d[name] = t[p:p + n]
        p += n
    assert p == len(t)
    return d


# ---------------------------------------------------------------------------------------
# launch descriptions, as csrc/engine.cu builds them
# ---------------------------------------------------------------------------------------

def causal_case(taus: list[int], n0: int, c: int, R: int) -> dict:
    """lag_causal: frames n0..n0+c-1 against every tau, windows in descending tau."""
    tmax, T = max(taus), len(taus)
    slot = lambda f: f % R if f >= 0 else -1  # noqa: E731
    return {"nreg": c, "reg": [slot(n0 + j) for j in range(c)],
            "ent_acc": list(range(T - 1, -1, -1)),
            "ent_w": [tmax - taus[i] for i in range(T - 1, -1, -1)],
            "pos": [slot(n0 - tmax + p) for p in range(c + tmax)]}


def compat_case(taus: list[int], start: list[int], end: list[int], f0: int, R: int) -> dict:
    """lag_iteration: A = start[f0..], partner of position q = start|end[q]."""
    C = len(start)
    nreg = min(64, C - f0)
    slot = lambda f: f % R if f >= 0 else -1  # noqa: E731
    pos = []
    for p in range(nreg + max(taus)):
        q = f0 + p
        lab = start[q] if q < C else (end[q - C] if q - C < C else -1)
        pos.append(slot(lab))
    return {"nreg": nreg, "reg": [slot(start[f0 + j]) for j in range(nreg)],
            "ent_acc": list(range(len(taus))), "ent_w": list(taus), "pos": pos}


def random_case(rnd: random.Random) -> dict:
    nreg = rnd.choice([1, 3, 4, 7, 8, 16, 20, 29, 30, 32, 33, 50, 63, 64])
    ntau = rnd.randint(1, 70)
    starts = sorted(rnd.sample(range(0, 600), ntau))
    npos = starts[-1] + nreg
    R = rnd.choice([40, 97, 530, 4096])
    base = rnd.randrange(R)
    hole = rnd.random() * 0.3
    pos = [-1 if rnd.random() < hole else (base + p) % R for p in range(npos)]
    reg = [-1 if rnd.random() < hole / 3 else rnd.randrange(R) for _ in range(nreg)]
    return {"nreg": nreg, "reg": reg, "ent_acc": [rnd.randrange(128) for _ in range(ntau)],
            "ent_w": starts, "pos": pos}


def schedule_cases() -> list[dict]:
    cases = []
    tau_sets = [log_taus(1, 500, 64), [1, 2, 3, 5, 8, 13, 21, 34, 55], list(range(1, 21)),
                log_taus(1, 300, 48), [1], [7, 300]]
    for taus in tau_sets:
        for c in (30, 32, 20, 8, 1, 3, 64, 60, 45):
            R = max(taus) + 63 + 2 * min(c, 64)
            for n0 in (0, 7, 30, 200, 600, 1000):
                cases.append(causal_case(taus, n0, c, R))
    for taus, C in ((list(range(1, 21)), 20), ([1, 2, 4, 8, 16, 32], 40), ([1, 3, 9], 10), ([2, 5], 64),
                    (log_taus(1, 500, 64), 500)):
        R = 3 * C + 5
        for base in (0, 7 * C):
            start = [base + i for i in range(C)]
            for end in ([base + C + i for i in range(C)], [-1] * C,            # tail: nothing yet
                        [base + 2 * C + i for i in range(C)]):                 # stale pinned buffer
                for f0 in range(0, C, 64):
                    cases.append(compat_case(taus, start, end, f0, R))
    rnd = random.Random(1234)
    cases += [random_case(rnd) for _ in range(150)]
    return cases


# ---------------------------------------------------------------------------------------
# checks
# ---------------------------------------------------------------------------------------

def check_table(case: dict, d: dict) -> None:
    nreg, J = case["nreg"], pick_j(case["nreg"])
    assert d["nreg"] == nreg and d["ntau"] == len(case["ent_acc"])
    assert d["reg"][:nreg] == case["reg"][:nreg] and all(v == -1 for v in d["reg"][nreg:])
    assert d["ent_acc"] == case["ent_acc"]
    nu, ub, us = d["nu"], d["ub"], d["uslot"]
    for e, w in enumerate(case["ent_w"]):
        assert 0 <= ub[e] and ub[e] + nreg <= nu
        if e:
            assert ub[e] > ub[e - 1]
        assert us[ub[e]:ub[e] + nreg] == case["pos"][w:w + nreg]
        full = nreg == J and all(r >= 0 for r in case["reg"][:nreg]) and all(s >= 0 for s in us[ub[e]:ub[e] + nreg])
        assert d["full"][e] & FULL_FLAG == int(full)
    # fused runs: greedy, FUSE full entries whose windows start one union entry apart
    e, starts = 0, set()
    while e + FUSE <= len(ub):
        if all(d["full"][e + r] & FULL_FLAG and ub[e + r] == ub[e] + r for r in range(FUSE)):
            starts.add(e)
            e += FUSE
        else:
            e += 1
    assert {e for e in range(len(ub)) if d["full"][e] & RUN_FLAG} == starts
    assert all(f & ~(FULL_FLAG | RUN_FLAG) == 0 for f in d["full"])
    # the union holds each window position once: its size is the number of distinct positions
    covered = set()
    for w in case["ent_w"]:
        covered.update(range(w, w + nreg))
    assert nu == len(covered)
    assert d["ngroups"] == (nu + GROUP - 1) // GROUP
    seen = set()
    for g in range(d["ngroups"]):
        for run in d["runs"][d["gptr"][g]:d["gptr"][g + 1]]:
            slot, rows, rel = run & 0xFFFFF, 1 << ((run >> 20) & 3), (run >> 22) & 7
            assert rel + rows <= GROUP
            for i in range(rows):
                u = g * GROUP + rel + i
                assert u < nu and us[u] == slot + i and u not in seen
                seen.add(u)
    assert seen == {u for u in range(nu) if us[u] >= 0}
    ntab = TAB_ENTRIES + 3 * d["ntau"] + nu + d["ngroups"] + 1 + len(d["runs"])
    slots = ring_slots(J)
    acc_ring = ACC_SLOTS * CONSUMERS * 32 * 8  # accumulator prefetch ring
    assert slots * slot_bytes(J) + 2 * 8 * (slots // GROUP) + acc_ring + 4 * (2 + ntab) <= SMEM_MAX


def parity_done(completed: int, parity: int) -> bool:
    """mbarrier try_wait.parity P returns once the phase with parity P has completed."""
    return completed >= 1 and (completed - 1) % 2 == parity


def replay(d: dict, seed: int, skip_empty_waits: bool = False, blocks: int = 1,
           one_block_slots: bool = False, consumers: int = CONSUMERS) -> str:
    """Random interleaving of the producer lane and the consumer warps, as lag_pipe_kernel
    walking ``blocks`` element blocks of one launch (its persistent grid): the producer issues
    group g of block n as running group G = n * ngroups + g into group slot G % slots; a
    consumer waits once per window for every group up to the window's last, reads the window
    (union entry u of block n sits in the slot of running group n * ngroups + u // 8), releases
    the groups below the next window, and at the end of a block waits for and releases every
    group of the block. ``skip_empty_waits`` and ``one_block_slots`` plant errors the kernel
    avoids: not waiting on groups without frames, and looking for union entry u of every
    block in the slot of group u // 8 (the rule for a single block). ``consumers`` is the
    number of consumer warps: 4 in the one-thread-per-element geometry, 8 in the
    two-threads-per-element one."""
    rnd = random.Random(seed)
    nreg, ntau, nu, ngroups, ub = d["nreg"], d["ntau"], d["nu"], d["ngroups"], d["ub"]
    gslots = ring_slots(pick_j(nreg)) // GROUP
    empty_groups = {g for g in range(ngroups) if d["gptr"][g] == d["gptr"][g + 1]}
    full_c, empty_c, empty_arr = [0] * gslots, [0] * gslots, [0] * gslots
    content = [None] * gslots  # which running group a group slot holds
    g_next = 0
    warps = [{"b": 0, "e": 0, "waited": 0, "released": 0} for _ in range(consumers)]

    def landed(base: int, groups) -> bool:
        return all(parity_done(full_c[(base + g) % gslots], ((base + g) // gslots) & 1) for g in groups
                   if not (skip_empty_waits and g in empty_groups))

    def release(s: dict, base: int, upto: int) -> None:
        for g in range(s["released"], upto):
            gs = (base + g) % gslots
            empty_arr[gs] += 1
            if empty_arr[gs] == consumers:
                empty_arr[gs] = 0
                empty_c[gs] += 1
        s["released"] = max(s["released"], upto)

    idle = 0
    while True:
        actors = (["P"] if g_next < blocks * ngroups else []) + [w for w in range(consumers) if warps[w]["b"] < blocks]
        if not actors:
            return "ok"
        a = rnd.choice(actors)
        progressed = False
        if a == "P":
            gs, fill = g_next % gslots, g_next // gslots
            if fill == 0 or parity_done(empty_c[gs], (fill - 1) & 1):
                full_c[gs] += 1  # data landed (or bare arrive for a group without frames)
                content[gs] = g_next
                g_next += 1
                progressed = True
        else:
            s = warps[a]
            base = s["b"] * ngroups
            e = s["e"]
            if e == ntau:  # end of the block: every group waited for and released
                if landed(base, range(s["waited"], ngroups)):
                    release(s, base, ngroups)
                    s.update(b=s["b"] + 1, e=0, waited=0, released=0)
                    progressed = True
            else:
                nrun = FUSE if d["full"][e] & RUN_FLAG else 1  # a fused run waits once for its span
                glast = (ub[e + nrun - 1] + nreg - 1) // GROUP
                if landed(base, range(s["waited"], glast + 1)):
                    s["waited"] = max(s["waited"], glast + 1)
                    for r in range(nrun):
                        for j in range(nreg):
                            u = ub[e + r] + j
                            slot = (u // GROUP if one_block_slots else base + u // GROUP) % gslots
                            if d["uslot"][u] >= 0 and d["reg"][j] >= 0 and content[slot] != base + u // GROUP:
                                return f"stale read of union entry {u} by entry {e + r} of block {s['b']}"
                    s["e"] += nrun
                    release(s, base, ub[s["e"]] // GROUP if s["e"] < ntau else ngroups)
                    progressed = True
        idle = 0 if progressed else idle + 1
        if idle > 4000:
            return "deadlock"


def test_tables_and_protocol(probe):
    cases = schedule_cases()
    tables = build_tables(probe, cases)
    for i, (case, t) in enumerate(zip(cases, tables)):
        assert not isinstance(t, str), (i, t)
        d = parse(t)
        check_table(case, d)
        for seed in range(2):
            assert replay(d, seed) == "ok", (i, seed)
            assert replay(d, seed, blocks=3) == "ok", (i, seed)
        if d["nreg"] <= 32:  # the two-threads-per-element geometry: eight consumer warps
            assert replay(d, 0, blocks=3, consumers=8) == "ok", i


def test_windows_must_ascend(probe):
    case = causal_case([1, 2, 3], 10, 4, 20)
    case["ent_w"] = case["ent_w"][::-1]
    assert build_tables(probe, [case])[0] == "ERR lag windows out of order"


def test_union_shrinks_reads():
    """The union is what makes the kernel read fewer bytes than one frame per pair: a
    30-frame chunk against 64 log-spaced taus up to 500 needs 484 partner frames, not 1920."""
    taus = log_taus(1, 500, 64)
    case = causal_case(taus, 1000, 30, 560)
    covered = set()
    for w in case["ent_w"]:
        covered.update(range(w, w + 30))
    assert len(covered) == 484


def test_wrong_protocol_is_caught(probe):
    """The replay catches a consumer that skips waiting on groups without frames (the
    protocol error the kernel avoids): it may then release a group slot before the producer
    has filled it, which shows up as a stale read or a deadlock."""
    for c in (30, 64):
        d = parse(build_tables(probe, [causal_case(log_taus(1, 500, 64), 0, c, 700)])[0])
        assert any(d["gptr"][g] == d["gptr"][g + 1] for g in range(d["ngroups"])), "needs frame-less groups"
        assert any(replay(d, seed, skip_empty_waits=True) != "ok" for seed in range(20))
        assert all(replay(d, seed) == "ok" for seed in range(20))


def test_ring_must_hold_a_full_window(probe, monkeypatch):
    """With 64 register frames a 64-slot ring cannot hold a window and the group the next
    window shares with it: the replay deadlocks, which is why that kernel has 128 slots."""
    d = parse(build_tables(probe, [causal_case(list(range(1, 21)), 200, 64, 200)])[0])
    assert replay(d, 0) == "ok"
    monkeypatch.setattr(sys.modules[__name__], "ring_slots", lambda J: 64)
    assert replay(d, 0) == "deadlock"


def test_block_offset_is_needed(probe):
    """Over several element blocks a group of block n lands in the slot of running group
    n * ngroups + g: a consumer that looked for union entry u in slot u // 8 (the one-block
    rule) reads other groups' data whenever ngroups is not a multiple of the group slots."""
    d = parse(build_tables(probe, [causal_case(log_taus(1, 500, 64), 1000, 32, 700)])[0])
    assert d["ngroups"] % (ring_slots(32) // GROUP) != 0
    assert replay(d, 0, blocks=3) == "ok"
    assert replay(d, 0, blocks=1, one_block_slots=True) == "ok"
    assert replay(d, 0, blocks=3, one_block_slots=True).startswith("stale read")
