"""Generate tests/golden/tutorial1_topology.npz from the reference's own test fixture.

The reference's only test (tests/Tutorial_1) ships the Triangle mesh-generator outputs
iRICZone.1.edge (edge endpoints + boundary marker) and iRICZone.1.v.edge (the two
triangles of each edge; -1 marks a Voronoi ray, i.e. a boundary edge) next to its
CGNS case.  The node coordinates live only in Case1.cgn (HDF5, no reader here), so the
fixture keeps the topology: edges, their element pairs, the boundary markers and the
triangles rebuilt from the edges with one consistent orientation.

Run from the repository root, naming the reference checkout's Tutorial_1 folder:
    python tests/golden/make_tutorial1_fixture.py <reference>/tests/Tutorial_1
(or set STORM_TUTORIAL1_DIR to that folder).
"""
import collections
import os
import sys

import numpy as np

OUT = os.path.join(os.path.dirname(os.path.abspath(__file__)), "tutorial1_topology.npz")


def read_table(path, ncol):
    rows = []
    with open(path) as f:
        n = int(f.readline().split()[0])
        for _ in range(n):
            rows.append([float(x) for x in f.readline().split()[:ncol]])
    return np.array(rows)


def main():
    src = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("STORM_TUTORIAL1_DIR")
    if not src:
        sys.exit("usage: make_tutorial1_fixture.py <reference>/tests/Tutorial_1")
    e = read_table(os.path.join(src, "iRICZone.1.edge"), 4).astype(np.int64)
    v = read_table(os.path.join(src, "iRICZone.1.v.edge"), 3).astype(np.int64)
    assert np.array_equal(e[:, 0], np.arange(1, len(e) + 1))
    assert np.array_equal(v[:, 0], np.arange(1, len(v) + 1))
    edge_p = e[:, 1:3]
    marker = e[:, 3]
    edge_e = v[:, 1:3]
    ntri = int(edge_e.max())
    tri_edges = collections.defaultdict(list)
    for k, (a, b) in enumerate(edge_e):
        for t in (a, b):
            if t > 0:
                tri_edges[t].append(k)
    assert len(tri_edges) == ntri and all(len(x) == 3 for x in tri_edges.values())
    # orient every triangle, then make orientations consistent across shared edges
    tri = np.zeros((ntri, 3), dtype=np.int64)
    for t in range(1, ntri + 1):
        ks = sorted(tri_edges[t])
        a, b = edge_p[ks[0]]
        verts = set(edge_p[ks[0]]) | set(edge_p[ks[1]]) | set(edge_p[ks[2]])
        (c,) = verts - {a, b}
        tri[t - 1] = (a, b, c)
    def directed(t):
        a, b, c = tri[t - 1]
        return {(a, b), (b, c), (c, a)}
    seen = np.zeros(ntri + 1, dtype=bool)
    for root in range(1, ntri + 1):
        if seen[root]:
            continue
        seen[root] = True
        stack = [root]
        while stack:
            t = stack.pop()
            dt = directed(t)
            for k in tri_edges[t]:
                for s in edge_e[k]:
                    if s <= 0 or s == t or seen[s]:
                        continue
                    p, q = edge_p[k]
                    same = ((p, q) in dt) == ((p, q) in directed(s))
                    if same:  # must traverse the shared edge in opposite directions
                        tri[s - 1, 1], tri[s - 1, 2] = tri[s - 1, 2], tri[s - 1, 1]
                    seen[s] = True
                    stack.append(s)
    np.savez_compressed(OUT, edge_p=edge_p.astype(np.int32), edge_e=edge_e.astype(np.int32),
                        marker=marker.astype(np.int8), tri=tri.astype(np.int32),
                        n_pts=np.int32(edge_p.max()))
    print(OUT, os.path.getsize(OUT), "bytes;", "nodes", edge_p.max(), "tris", ntri, "edges", len(edge_p),
          "boundary", int((edge_e[:, 1] < 0).sum()), file=sys.stderr)


if __name__ == "__main__":
    main()
