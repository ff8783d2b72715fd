import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200, sm_100a)")
    config.addinivalue_line("markers", "slow: long-running CPU test")


def pytest_terminal_summary(terminalreporter):
    """The achieved GPU-vs-oracle errors of every parity assertion of the run."""
    import json

    from parity import RECORDS
    if not RECORDS:
        return
    tr = terminalreporter
    tr.write_sep("-", f"parity: achieved errors ({len(RECORDS)} assertions)")
    tr.write_line(f"{'label':44s} {'rel_E':>9s} {'floor_E':>9s} {'rel_F':>9s} {'floor_F':>9s}  fixed bars")
    for r in RECORDS:
        tr.write_line(f"{r['label'][:44]:44s} {r['rel_e']:9.2e} {r['floor_e']:9.2e} {r['rel_f']:9.2e} "
                      f"{r['floor_f']:9.2e}  {'yes' if r['fixed_bars_hold'] else 'no (floor)'}")
    path = os.environ.get("MDG_PARITY_LOG")
    if path:
        with open(path, "a") as f:
            for r in RECORDS:
                f.write(json.dumps(r) + "\n")
