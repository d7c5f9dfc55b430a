"""Writes join_digests.json: the expected summaries of the reference's join tests.

Usage: python make_golden.py <reference checkout>. The expected values are read from the
reference's test file, where they are written as literals (tests/python/test_package.py:2079-2113).
"""
from __future__ import annotations

import json
import os
import re
import sys

def main():
    if len(sys.argv) != 2:
        sys.exit("usage: python make_golden.py <reference checkout>")
    text = open(os.path.join(sys.argv[1], "tests/python/test_package.py")).read()
    entry = r"\((\d+), (\d+), ([0-9.]+), \"([0-9a-f]{16})\"\)"
    single = re.search(r"parametrize\(\"axis,digest\", \[(.*?)\]\)", text).group(1)
    out = {}
    for axis, dig in re.findall(r"\((\d), \"([0-9a-f]{16})\"\)", single):
        out[f"band_axis{axis}"] = {"1": [162, 161, 8.0, dig]}
    block = re.search(r"labels, expected, options = \{(.*?)\}\[case\]", text, re.S).group(1)
    for case, body in re.findall(r"\"(bands|wide|spiral)\": \((.*?)\}, \{", block, re.S):
        out[case] = {lab: [int(a), int(b), float(c), d] for lab, (a, b, c, d) in
                     ((m[0], m[1:]) for m in re.findall(r"(\d+): " + entry, body))}
    helix = re.search(r"_helix_tube\(1\.9, 8\.0, 28\.0, 28\), \{1: " + entry, text)
    out["helix"] = {"1": [int(helix.group(1)), int(helix.group(2)), float(helix.group(3)), helix.group(4)]}
    path = os.path.join(os.path.dirname(os.path.abspath(__file__)), "join_digests.json")
    with open(path, "w") as f:
        json.dump(out, f, indent=1, sort_keys=True)
    print(json.dumps(out, indent=1, sort_keys=True))


if __name__ == "__main__":
    main()
