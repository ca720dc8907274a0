"""Object BVH over Triangle objects (the CPU structure `Mesh` owns).

Same construction rule as the reference's core/bvh.py BVHNode: leaves of at
most `max_leaf_size` triangles (or depth > 20), otherwise the triangles are
stably sorted by centroid along the longest axis of their bounds (each
triangle's box padded by 1e-4) and split at the middle.  The root-level sort
reorders the caller's list in place, which fixes the order in which a Mesh's
triangles reach the GPU scene.  Ray queries on the GPU path use the device
LBVH built by libroxy_cuda.so instead of this tree.
"""

_EPS = 1e-4


def _bounds(triangles):
    lo = [float("inf")] * 3
    hi = [float("-inf")] * 3
    for t in triangles:
        for v in (t._v0, t._v1, t._v2):
            for k in range(3):
                lo[k] = min(lo[k], v[k] - _EPS)
                hi[k] = max(hi[k], v[k] + _EPS)
    return lo, hi


def _longest_axis(lo, hi):
    ex, ey, ez = hi[0] - lo[0], hi[1] - lo[1], hi[2] - lo[2]
    if ex >= ey and ex >= ez:
        return 0
    return 1 if ey >= ez else 2


def _centroid(t, axis):
    c = (t._v0 + t._v1 + t._v2) / 3.0
    return c[axis]


class BVHNode:
    def __init__(self, triangles, depth=0, max_leaf_size=4):
        self.bounds = _bounds(triangles)
        if len(triangles) <= max_leaf_size or depth > 20:
            self.triangles = triangles
            self.left = self.right = None
        else:
            axis = _longest_axis(*self.bounds)
            triangles.sort(key=lambda t: _centroid(t, axis))
            mid = len(triangles) // 2
            self.left = BVHNode(triangles[:mid], depth + 1)
            self.right = BVHNode(triangles[mid:], depth + 1)
            self.triangles = None

    def __repr__(self):
        if self.triangles is not None:
            return f"BVHNode(leaf, num_triangles={len(self.triangles)})"
        return f"BVHNode(interior, left={self.left}, right={self.right})"
