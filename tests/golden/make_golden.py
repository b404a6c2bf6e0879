"""Generate the byte-format golden fixtures with the reference's own converter.

Run in a checkout where the reference sources are available and
``make -C oracle ref`` has built ``oracle/_ref/converter`` and
``oracle/_ref/converter_weighted`` from converter/converter.cpp.  Writes:

  toy_edges.txt      text edge list "src dst weight" (duplicates, self-loops,
                     a zero-out-degree vertex and an isolated top id)
  toy.csr / toy.csc / toy.wcsr   converter --type csr|csc|wcsr (weight 20)
  toy_w.csr          converter built with -DWEIGHTED (weights from column 3)

The converter names its WCSR output "<base>..wcsr" (converter.cpp:777); it is
renamed to toy.wcsr here.
"""
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
REF = os.path.join(ROOT, "oracle", "_ref")


def edges():
    # deterministic mix: chains, a hub, duplicates, self-loops
    out = []
    for i in range(40):
        out.append((i, (i * 7 + 3) % 41, 1 + (i * 13) % 64))
    for j in range(1, 30, 3):
        out.append((5, j, 1 + j % 64))
    out += [(3, 3, 9), (7, 7, 2), (10, 11, 4), (10, 11, 4), (10, 11, 4)]
    out += [(44, 2, 17)]  # vertex 44: max id; 41..43 have no edges
    return out


def main():
    txt = os.path.join(HERE, "toy_edges.txt")
    with open(txt, "w") as f:
        for s, d, w in edges():
            f.write(f"{s} {d} {w}\n")
    tmp = os.path.join(HERE, "_tmp")
    os.makedirs(tmp, exist_ok=True)
    for kind, exe, out in [("csr", "converter", "toy.csr"), ("csc", "converter", "toy.csc"),
                           ("wcsr", "converter", "toy.wcsr"), ("csr", "converter_weighted", "toy_w.csr")]:
        src = os.path.join(tmp, "g.txt")
        shutil.copy(txt, src)
        subprocess.run([os.path.join(REF, exe), "--input", src, "--skip", "0", "--type", kind],
                       check=True, stdout=subprocess.DEVNULL)
        produced = {"csr": "g.csr", "csc": "g.csc", "wcsr": "g..wcsr"}[kind]
        shutil.move(os.path.join(tmp, produced), os.path.join(HERE, out))
    shutil.rmtree(tmp)
    print("wrote fixtures to", HERE)


if __name__ == "__main__":
    sys.exit(main())
