"""Regenerates the golden fixtures of this directory from the reference tree.

    python tests/golden/make_golden.py [REFERENCE_TREE]

Reads, from the reference project (fvella/EGSolver):
  script/clique_500_cp4.txt.gz   2000-vertex game (1,746,500 edges, weights +-1)
  script/sol.txt                 its solution as printed by the reference
                                 (`egsolver --input clique_500_cp4.txt.gz --eg0
                                 --cpu`, lines 43-2043 "ext)<TAB>credit")
  script/multi/eg_fig2.txt       5-vertex example game (no expected output
                                 ships with it)
  dataset/test/modelchecking/IEEE1394nparties=2_datasize=2_headersize=2_
  acksize=2_property4.mpg.gz     a 571,378-vertex game from model checking
                                 (no expected output ships with it)

and writes:
  clique_500_cp4.txt.gz   the same game re-serialised by this library's
                          writer (same vertices, owners, edge order, weights)
  clique_500_cp4.sol      "ext credit" per vertex, from sol.txt
  eg_fig2.txt             the example game, re-serialised
  ref_eg_fig2*.txt        the example game and the reference's shipped
                          copies of it (script/multi: 2 copies, 4 copies, 2
                          copies of 2 copies), byte for byte
  eg_fig2.sol             its credits, [0, 3, TOP, 0, TOP] for vertices 0..4:
                          derived by hand and confirmed by running the
                          reference's own driver (oracle/_ref/egsolver --cpu)
  ieee1394_p4.txt.gz      the model-checking game, re-serialised
  ieee1394_p4.sol.gz      "ext credit" per vertex as printed by the
                          reference's own driver (oracle/_ref/egsolver --cpu
                          --eg, built by `make -C oracle ref`)

The fixtures are committed; the GPU box has no reference tree.
"""
from __future__ import annotations

import gzip
import os
import subprocess
import sys
from pathlib import Path

HERE = Path(__file__).resolve().parent
sys.path.insert(0, str(HERE.parents[1]))

import egsolver_b200 as eg  # noqa: E402


def parse_solution(text: str) -> list[tuple[int, int]]:
    out = []
    in_sol = False
    for line in text.splitlines():
        if line.startswith("Solution:"):
            in_sol = True
            continue
        if in_sol and ")" in line and line.split(")")[0].strip().isdigit():
            k, v = line.split(")")
            out.append((int(k), int(v.strip())))
    return out


def main(ref: Path) -> None:
    game = eg.read_game(str(ref / "script" / "clique_500_cp4.txt.gz"))
    eg.write_game_text(game, str(HERE / "clique_500_cp4.txt.gz"))
    sol = parse_solution((ref / "script" / "sol.txt").read_text())
    assert len(sol) == 2000, len(sol)
    (HERE / "clique_500_cp4.sol").write_text("".join(f"{k} {v}\n" for k, v in sorted(sol)))
    fig = eg.read_game(str(ref / "script" / "multi" / "eg_fig2.txt"))
    (HERE / "eg_fig2.txt").write_text(eg.game_to_text(fig))
    # the example game and the reference's own multi outputs of it, verbatim
    # (byte-level fixtures of the copies generator)
    for name in ("eg_fig2", "eg_fig2_duecopie", "eg_fig2_quattrocopie", "eg_fig2_duecopie_di_duecopie"):
        (HERE / f"ref_{name}.txt").write_bytes((ref / "script" / "multi" / f"{name}.txt").read_bytes())
    top = 2147483647
    (HERE / "eg_fig2.sol").write_text("".join(f"{k} {v}\n" for k, v in enumerate([0, 3, top, 0, top])))
    mc = ref / "dataset" / "test" / "modelchecking" / (
        "IEEE1394nparties=2_datasize=2_headersize=2_acksize=2_property4.mpg.gz")
    eg.write_game_text(eg.read_game(str(mc)), str(HERE / "ieee1394_p4.txt.gz"))
    drv = HERE.parents[1] / "oracle" / "_ref" / "egsolver"
    out = subprocess.run([str(drv), "--cpu", "--eg", "--input", str(mc)], capture_output=True, text=True,
                         check=True, timeout=3600).stdout
    sol = parse_solution(out)
    assert len(sol) == 571378, len(sol)
    with gzip.open(HERE / "ieee1394_p4.sol.gz", "wt") as f:
        f.write("".join(f"{k} {v}\n" for k, v in sorted(sol)))
    print("wrote fixtures to", HERE)


if __name__ == "__main__":
    # the reference checkout: argv[1], $EG_REFERENCE_TREE, else "reference" beside this repository
    default = os.environ.get("EG_REFERENCE_TREE", str(HERE.parents[2] / "reference"))
    main(Path(sys.argv[1]) if len(sys.argv) > 1 else Path(default))
