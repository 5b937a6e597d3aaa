"""The binomial checkpointing schedule (dasha_b200/csrc/checkpoint_schedule.h) on the host: a
simulator replays its actions and checks that every step is reversed once, in order n-1 .. 0,
from its own state, within the slots given; the forward steps it takes equal the closed-form
cost, which equals the optimum of the recursion computed here by dynamic programming."""
import functools
import os
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
DRIVER = r'''
#include "checkpoint_schedule.h"
#include <cstdio>
#include <cstdlib>
int main(int argc, char** argv) {
    if (argv[1][0] == 'c') {                       // c n s: the closed-form cost
        std::printf("%lld\n", dasha::binomial_cost(std::atoll(argv[2]), std::atoll(argv[3])));
        return 0;
    }
    for (const auto& a : dasha::binomial_schedule(std::atoi(argv[2]), std::atoi(argv[3])))
        std::printf("%d %d %d\n", a.kind, a.a, a.b);
    return 0;
}
'''


@pytest.fixture(scope="module")
def driver(tmp_path_factory):
    d = tmp_path_factory.mktemp("ckpt")
    src, exe = d / "drv.cpp", d / "drv"
    src.write_text(DRIVER)
    subprocess.run(["g++", "-O2", "-std=c++17", "-I", os.path.join(ROOT, "dasha_b200", "csrc"), str(src), "-o", str(exe)],
                   check=True)
    return str(exe)


def schedule(driver, n, s):
    out = subprocess.run([driver, "s", str(n), str(s)], capture_output=True, text=True, check=True).stdout
    return [tuple(map(int, line.split())) for line in out.splitlines()]


def cost(driver, n, s):
    return int(subprocess.run([driver, "c", str(n), str(s)], capture_output=True, text=True, check=True).stdout)


@functools.lru_cache(maxsize=None)
def dp(l, s):
    if l <= 1:
        return 0
    if s == 0:
        return l * (l - 1) // 2
    return min(m + dp(l - m, s - 1) + dp(m, s) for m in range(1, l))


def simulate(actions, n, s):
    """Replays the actions; returns the forward steps taken."""
    RESTORE, ADVANCE, STORE, RELEASE, REVERSE = range(5)
    slots = {0: 0}                 # slot -> step whose state it holds
    current, steps, reversed_ = 0, 0, []
    for kind, a, b in actions:
        if kind == RESTORE:
            assert a in slots and slots[a] == b
            current = b
        elif kind == ADVANCE:
            assert current == a and b > a
            steps += b - a
            current = b
        elif kind == STORE:
            assert current == b and a not in slots and 1 <= a <= s
            slots[a] = b
        elif kind == RELEASE:
            assert slots.get(a) == b and a != 0
            del slots[a]
        elif kind == REVERSE:
            assert current == a
            reversed_.append(a)
            current = None         # the reverse sweep consumes the state
        assert len(slots) <= s + 1
    assert reversed_ == list(range(n - 1, -1, -1))
    return steps


def test_closed_form_is_the_optimum(driver):
    for s in range(0, 5):
        for l in range(1, 41):
            assert cost(driver, l, s) == dp(l, s), (l, s)


@pytest.mark.parametrize("n,s", [(1, 0), (2, 0), (7, 0), (10, 1), (25, 2), (40, 3), (100, 4), (500, 10), (500, 3), (64, 63)])
def test_schedule_is_valid_and_optimal(driver, n, s):
    steps = simulate(schedule(driver, n, s), n, s)
    assert steps == cost(driver, n, s)
    if n <= 40 and s <= 4:
        assert steps == dp(n, s)


def test_large_cases_closed_form(driver):
    """500 steps: with 11 states (slot 0 and 10 more, what fits beside the adjoint's scratch on
    a 512x256x512 FP64 grid) the schedule takes 1545 forward steps, 3.1 runs, where two-level
    checkpointing needs about 45 states; with 4 states 3213; with every state kept (499 more
    slots) one sweep, 499 steps; with 46 states, the memory of two-level checkpointing, 952."""
    assert cost(driver, 500, 3) == 3213
    assert cost(driver, 500, 10) == 1545
    assert cost(driver, 500, 499) == 499
    assert cost(driver, 500, 45) == 952
