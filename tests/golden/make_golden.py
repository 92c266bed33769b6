"""Extract the reference's frozen b155550 trajectories into ``tests/golden/b155550.json``.

Run once where the reference tree is present, naming its root:

    python tests/golden/make_golden.py <reference-root>

It copies numbers only (S^z profiles, bond dimensions, statuses, errors against the exact answer,
the discarded weight, norms and the no-symmetry final state) from
``test/fixtures/b155550/{xx_u1_bug_order1,xx_u1_bug_order2,xx_none_bug_order2}.json`` (read by the
reference's ``test/BUG/TimeEvolution/test_fixtures_b155550.jl``) and the two-site TDVP baseline's
``baseline_tdvp2_xx.json`` (read by ``test/Baselines/test_baselines.jl``) and the imaginary-time
``heisenberg_ite.json`` (read by ``test_fixtures_b155550.jl`` as well), and the Heston backward
pricing run ``qtt_heston_backward.json`` (read by ``test/QTTS/Tooling/test_nonlinear_step.jl``:
its final 5 + 5-bit state and bond dimensions).
"""

import json
import pathlib
import sys


def main(ref_root: str) -> None:
    src = pathlib.Path(ref_root) / "test" / "fixtures" / "b155550"
    out = {"source": "test/fixtures/b155550", "versions": json.load(open(src / "versions.json"))}
    for name in ("xx_u1_bug_order1", "xx_u1_bug_order2", "xx_none_bug_order2", "baseline_tdvp2_xx",
                 "heisenberg_ite", "qtt_heston_backward"):
        d = json.load(open(src / f"{name}.json"))
        d.pop("wall_s", None)
        out[name] = d
    dst = pathlib.Path(__file__).with_name("b155550.json")
    dst.write_text(json.dumps(out, indent=1))
    print("wrote", dst)


if __name__ == "__main__":
    if len(sys.argv) != 2:
        sys.exit("usage: make_golden.py <reference-root>")
    main(sys.argv[1])
