"""Host-side readers of the binary BVH layout (16 floats per node: child 0
box at columns 0-3 (x, y) and 8-9 (z), child 1 at 4-7 and 10-11, child links
as int bits at 12-13; a link < 0 is a leaf ~((first << 3) | (count - 1)) into
the leaf-order triangle array)."""
import numpy as np

BOX_COLS = ((0, 1, 2, 3, 8, 9), (4, 5, 6, 7, 10, 11))


def _leaf(code):
    v = ~int(code)
    return v >> 3, (v & 7) + 1


def canonical(nodes, ids):
    """Depth-first walk from the root, child 0 first: per child its six box
    floats as uint32 bits and, for a leaf, the sorted triangle ids. Two trees
    with the same splits, leaves and boxes give equal lists whatever their node
    numbering and in-leaf order."""
    bits = nodes.view(np.uint32)
    links = nodes[:, 12:14].view(np.int32)
    out = []
    stack = [0]
    while stack:
        n = stack.pop()
        kids = []
        for s in (0, 1):
            box = tuple(int(b) for b in bits[n, list(BOX_COLS[s])])
            c = int(links[n, s])
            if c < 0:
                first, count = _leaf(c)
                out.append((box, tuple(sorted(int(t) for t in ids[first:first + count]))))
            else:
                out.append((box, c >= 0))
                kids.append(c)
        stack.extend(reversed(kids))
    return out


def leaf_orders(nodes, ids):
    """Every leaf's triangle ids in stored order (sorted by the first id)."""
    links = nodes[:, 12:14].view(np.int32)
    out = []
    stack = [0]
    while stack:
        n = stack.pop()
        for s in (0, 1):
            c = int(links[n, s])
            if c < 0:
                first, count = _leaf(c)
                out.append(tuple(int(t) for t in ids[first:first + count]))
            else:
                stack.append(c)
    return sorted(set(out))


def validate(nodes, ids, vertices, indices):
    """Checks a tree on its own: every triangle in exactly one leaf, every
    child box holding its subtree, depth. Returns (inner nodes, depth)."""
    nt = indices.shape[0]
    assert sorted(ids.tolist()) == list(range(nt)), "leaf order is not a permutation of the triangles"
    tri = vertices[indices]  # (nt, 3, 3)
    tlo, thi = tri.min(axis=1), tri.max(axis=1)
    links = nodes[:, 12:14].view(np.int32)
    seen = np.zeros(nt, np.int32)

    def box(n, s):
        b = nodes[n, list(BOX_COLS[s])]
        return np.array([b[0], b[2], b[4]]), np.array([b[1], b[3], b[5]])

    inner, depth = 0, 0
    stack = [(0, None, 1)]
    while stack:
        n, outer, d = stack.pop()
        inner += 1
        depth = max(depth, d)
        for s in (0, 1):
            lo, hi = box(n, s)
            c = int(links[n, s])
            if outer is not None and lo[0] <= hi[0]:
                assert np.all(lo >= outer[0]) and np.all(hi <= outer[1]), "child box outside its parent's"
            if c < 0:
                first, count = _leaf(c)
                t = ids[first:first + count]
                if lo[0] <= hi[0]:
                    assert np.all(tlo[t] >= lo) and np.all(thi[t] <= hi), "triangle outside its leaf box"
                if n == 0 and s == 1 and lo[0] > hi[0]:
                    continue  # the empty second slot of a one-leaf tree
                seen[t] += 1
                depth = max(depth, d + 1)
            else:
                stack.append((c, (lo, hi), d + 1))
    assert np.all(seen == 1), "a triangle is in %s leaves" % sorted(set(seen.tolist()) - {1})
    return inner, depth
