import json
import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200) and the built libdasha.so")


@pytest.fixture(scope="session")
def oracle_mod():
    from oracle import oracle
    oracle.load()
    return oracle


# Figures measured by the configuration tests (errors, rates, ratios), printed in the terminal
# summary at the end of the run so that they show in the tail of a quiet pytest run.
FIGURES = []


@pytest.fixture
def report():
    def add(name, **values):
        FIGURES.append((name, values))
    return add


def pytest_terminal_summary(terminalreporter):
    if FIGURES:
        terminalreporter.section("measured figures")
        for name, values in FIGURES:
            terminalreporter.write_line(f"{name}: {json.dumps(values, default=float)}")
