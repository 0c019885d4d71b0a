"""Write square_quads.msh: a 3 x 2 quad mesh of the unit square in Gmsh 2.2
ASCII, for the problem-file tests. Cell set 1 is the left column, 2 the
rest; face sets 10 bottom, 11 right, 12 top, 13 left.

    python tests/golden/problems/make_square_quads.py
"""
import os

HERE = os.path.dirname(os.path.abspath(__file__))


def main():
    nx, ny = 3, 2
    nodes = [(i / nx, j / ny) for j in range(ny + 1) for i in range(nx + 1)]
    nid = lambda i, j: j * (nx + 1) + i + 1
    lines = []
    for i in range(nx):
        lines.append((10, [nid(i, 0), nid(i + 1, 0)]))
        lines.append((12, [nid(i + 1, ny), nid(i, ny)]))
    for j in range(ny):
        lines.append((11, [nid(nx, j), nid(nx, j + 1)]))
        lines.append((13, [nid(0, j + 1), nid(0, j)]))
    quads = [(1 if i == 0 else 2, [nid(i, j), nid(i + 1, j), nid(i + 1, j + 1), nid(i, j + 1)])
             for j in range(ny) for i in range(nx)]
    out = ["$MeshFormat", "2.2 0 8", "$EndMeshFormat", "$PhysicalNames", "6",
           '1 10 "bottom"', '1 11 "right"', '1 12 "top"', '1 13 "left"', '2 1 "column"', '2 2 "rest"',
           "$EndPhysicalNames", "$Nodes", str(len(nodes))]
    out += [f"{k + 1} {x:.17g} {y:.17g} 0" for k, (x, y) in enumerate(nodes)]
    out += ["$EndNodes", "$Elements", str(len(lines) + len(quads))]
    k = 1
    for tag, vs in lines:
        out.append(f"{k} 1 2 {tag} {tag} " + " ".join(map(str, vs)))
        k += 1
    for tag, vs in quads:
        out.append(f"{k} 3 2 {tag} {tag} " + " ".join(map(str, vs)))
        k += 1
    out.append("$EndElements")
    with open(os.path.join(HERE, "square_quads.msh"), "w") as f:
        f.write("\n".join(out) + "\n")


if __name__ == "__main__":
    main()
