"""Extracts the reference's lane lockstep fixture into
tests/golden/chain_deck.json: the 8-stage inverter chain deck with RC wires
and its 19 rows of (wn, wp, rw, cw, td) from src/tests/espice.zig
(`chain_deck` :3072-3103, `chain_rows` :3110-3122), the deck with its .data
table and sweep removed so the rows come in as points. The reference test
runs each row alone and in three orders and asserts the same measures; the
tests run the rows as lanes on the GPU and through the oracle. Run from the
repository root with the path of the reference's source tree:

    python tests/golden/extract_chain_deck.py <reference tree>
"""
import json
import os
import re
import sys

OUT = os.path.join(os.path.dirname(os.path.abspath(__file__)), "chain_deck.json")


def main(tree: str):
    text = open(os.path.join(tree, "src", "tests", "espice.zig")).read().splitlines()
    start = next(i for i, l in enumerate(text) if l.startswith("const chain_deck ="))
    deck = []
    for line in text[start + 1:]:
        s = line.strip()
        if not s.startswith("\\\\"):
            break
        deck.append(s[2:])
    body = "\n".join(deck) + "\n"
    # the .data table and the sweep go; the rows become points
    body = re.sub(r"\.data pts.*?\.enddata\n", "", body, flags=re.S).replace(" sweep data=pts", "")
    rstart = next(i for i, l in enumerate(text) if l.startswith("const chain_rows"))
    rows_src = []
    for line in text[rstart + 1:]:
        if line.startswith("};"):
            break
        rows_src.append(line)
    rows = [[float(v) for v in m.split(",") if v.strip()]
            for m in re.findall(r"\.\{([^}]*)\}", "\n".join(rows_src))]
    assert len(rows) == 19 and all(len(r) == 5 for r in rows)
    json.dump({"source": "src/tests/espice.zig:3072-3122 (chain_deck, chain_rows)",
               "live": ["wn", "wp", "rw", "cw", "td"], "deck": body, "rows": rows},
              open(OUT, "w"), indent=1)


if __name__ == "__main__":
    if len(sys.argv) != 2:
        sys.exit("usage: extract_chain_deck.py <reference source tree>")
    main(sys.argv[1])
