"""Generate the golden per-tick digests of the oracle (test fixtures).

Run from the repository root: python tests/golden/make_golden.py
Each file holds, per tick, [state digest, FIFO digest, seed digest, last_tick_cells] of the
oracle (the CPU restatement of src/fluid.rs) on a synthetic workload.
"""
import json
import sys
from pathlib import Path

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT))
sys.path.insert(0, str(ROOT / "tests"))

import __graft_entry__ as ge  # noqa: E402
from conftest import oracle_for  # noqa: E402

CASES = [("basin_c1.json", 1, 1.0, 1, 300)]


def main():
    ge.build()
    vf, orc = ge.load_package(), ge.load_oracle()
    for name, wid, scale, seed, ticks in CASES:
        wl = vf.Workload(wid, scale, seed)
        o = oracle_for(orc, wl.world(0))
        for box in wl.wakes(0):
            o.wake(*map(int, box))
        digs = []
        for _ in range(ticks):
            o.tick()
            digs.append(list(o.digest()) + [o.last_tick_cells()])
        (ROOT / "tests" / "golden" / name).write_text(json.dumps({"workload": wid, "scale": scale, "seed": seed, "digests": digs}))
        print(name, ticks, "ticks")


if __name__ == "__main__":
    main()
