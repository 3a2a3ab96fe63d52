"""Golden vectors of the reference's own kernel fixtures, extracted for the
CPU pins (the reference tree is not present where the tests also run).

Reads ``tests/data/love_reference.txt`` (the Love cell integral of 1/|r-r'|
at 472 points, 80-digit arithmetic, columns x y a b value in units of h;
read by the reference's tests/test_kernel_stability.cpp:53-83) and
``tests/data/cerruti_reference.txt`` (the Cerruti kernel table read by
tests/test_cerruti.cpp) from the reference tree and writes their numeric rows
to ``tests/golden/love_reference.txt`` / ``cerruti_reference.txt`` with a
header naming the source.

Run: python tests/golden/make_reference_fixtures_txt.py [reference root]
"""

import os
import sys

HERE = os.path.dirname(os.path.abspath(__file__))


def extract(src, dst, what, root):
    rows = []
    header = None
    with open(src) as f:
        for line in f:
            if line.startswith("# x "):  # the column names
                header = line.strip()
            if line.startswith("#") or not line.strip():
                continue
            rows.append(line.split())
    with open(dst, "w") as f:
        f.write("# %s: numeric rows of the reference's %s\n" % (what, os.path.relpath(src, root)))
        if header:
            f.write(header + "\n")
        for r in rows:
            f.write(" ".join(r) + "\n")
    return len(rows)


if __name__ == "__main__":
    ROOT_REF = sys.argv[1] if len(sys.argv) > 1 else "/root/reference"
    n = extract(os.path.join(ROOT_REF, "tests", "data", "love_reference.txt"),
                os.path.join(HERE, "love_reference.txt"), "Love cell integral", ROOT_REF)
    m = extract(os.path.join(ROOT_REF, "tests", "data", "cerruti_reference.txt"),
                os.path.join(HERE, "cerruti_reference.txt"), "Cerruti kernel", ROOT_REF)
    print(n, m)
