"""Seeded synthetic scenes and cameras with the shapes of the benchmark workloads.

No dataset is available offline; these generators stand in for the reference's
scenes (GauUScene / UrbanScene aerial captures) with the stated sizes and
value distributions.  Camera conventions follow the reference
(LoG/dataset/base.py:20-55, LoG/utils/camera.py:4-29): OpenCV axes (x right,
y down, z forward), viewmatrix = [R|T]^T (world->view, transposed),
projmatrix = viewmatrix @ getProjectionMatrix2(K, H, W, near, far)^T,
tan_fov = W / (2 fx), H / (2 fy).  All arrays are numpy float32 / int32.
"""
import math

import numpy as np


# ---------------------------------------------------------------- cameras
def projection_matrix(fx, fy, cx, cy, W, H, znear, zfar):
    """getProjectionMatrix2 (LoG/utils/camera.py:7-29)."""
    P = np.zeros((4, 4), np.float32)
    P[0, 0] = 2 * fx / W
    P[0, 2] = -1 + 2 * (cx / W)
    P[1, 1] = 2 * fy / H
    P[1, 2] = -1 + 2 * (cy / H)
    P[2, 2] = zfar / (zfar - znear)
    P[2, 3] = -(zfar * znear) / (zfar - znear)
    P[3, 2] = 1.0
    return P


class Camera:
    """One pinhole view in the reference's raster-settings form."""

    def __init__(self, R, center, fx, fy, W, H, znear, zfar, cx=None, cy=None):
        R = np.asarray(R, np.float64)
        center = np.asarray(center, np.float64).reshape(3)
        T = -R @ center
        w2v = np.eye(4)
        w2v[:3, :3] = R
        w2v[:3, 3] = T
        self.W, self.H = int(W), int(H)
        self.fx, self.fy = float(fx), float(fy)
        cx = W / 2.0 if cx is None else cx
        cy = H / 2.0 if cy is None else cy
        proj = projection_matrix(fx, fy, cx, cy, W, H, znear, zfar).T.astype(np.float64)
        self.viewmatrix = w2v.T.astype(np.float32)                # world_view_transform
        self.projmatrix = (w2v.T @ proj).astype(np.float32)       # full_proj_transform
        self.campos = center.astype(np.float32)
        self.tanfovx = float(W / (2.0 * fx))
        self.tanfovy = float(H / (2.0 * fy))
        self.znear, self.zfar = znear, zfar

    def settings_kwargs(self):
        return dict(image_height=self.H, image_width=self.W, tanfovx=self.tanfovx, tanfovy=self.tanfovy,
                    viewmatrix=self.viewmatrix, projmatrix=self.projmatrix, campos=self.campos)


def look_rotation(forward, up=(0.0, 0.0, 1.0)):
    """World->camera rotation for an OpenCV camera looking along `forward`."""
    f = np.asarray(forward, np.float64)
    f = f / np.linalg.norm(f)
    r = np.cross(f, np.asarray(up, np.float64))
    if np.linalg.norm(r) < 1e-9:
        r = np.cross(f, np.array([0.0, 1.0, 0.0]))
    r = r / np.linalg.norm(r)
    d = np.cross(f, r)
    c2w = np.stack([r, d, f], axis=1)
    return c2w.T


def aerial_camera(rng, W=1920, H=1080, fx=1600.0, altitude=150.0, pitch_deg=45.0, xy_range=300.0, znear=0.1,
                  zfar=2000.0, yaw=None):
    yaw = rng.uniform(0, 2 * math.pi) if yaw is None else yaw
    pitch = math.radians(pitch_deg)
    center = np.array([rng.uniform(-xy_range, xy_range), rng.uniform(-xy_range, xy_range), altitude])
    fwd = np.array([math.cos(yaw) * math.cos(pitch), math.sin(yaw) * math.cos(pitch), -math.sin(pitch)])
    fy = fx
    return Camera(look_rotation(fwd), center, fx, fy, W, H, znear, zfar)


def look_at_camera(center, target, W=1920, H=1080, fx=1600.0, znear=0.1, zfar=2000.0):
    fwd = np.asarray(target, np.float64) - np.asarray(center, np.float64)
    return Camera(look_rotation(fwd), center, fx, fx, W, H, znear, zfar)


def identity_camera(W=256, H=256, fx=300.0, fy=300.0, znear=0.01, zfar=100.0):
    return Camera(np.eye(3), np.zeros(3), fx, fy, W, H, znear, zfar)


# ---------------------------------------------------------------- quaternions
def quat_mul(a, b):
    w1, x1, y1, z1 = a[..., 0], a[..., 1], a[..., 2], a[..., 3]
    w2, x2, y2, z2 = b[..., 0], b[..., 1], b[..., 2], b[..., 3]
    return np.stack([w1 * w2 - x1 * x2 - y1 * y2 - z1 * z2, w1 * x2 + x1 * w2 + y1 * z2 - z1 * y2,
                     w1 * y2 - x1 * z2 + y1 * w2 + z1 * x2, w1 * z2 + x1 * y2 - y1 * x2 + z1 * w2], axis=-1)


def random_unit_quats(rng, n):
    q = rng.standard_normal((n, 4))
    return (q / np.linalg.norm(q, axis=1, keepdims=True)).astype(np.float32)


def _sh(rng, n, degree=3):
    M = (degree + 1) ** 2
    sh = np.empty((n, M, 3), np.float32)
    sh[:, 0, :] = rng.normal(0, 0.5, (n, 3))
    sh[:, 1:, :] = rng.normal(0, 0.1, (n, M - 1, 3))
    return sh


def _sigmoid(x):
    return 1.0 / (1.0 + np.exp(-x))


# ---------------------------------------------------------------- scenes
def small_scene(P=10000, seed=1000, W=256, H=256, degree=3):
    """Camera-frame cube scene: P Gaussians, means U([-1,1]^2 x [2,6]), identity pose."""
    rng = np.random.default_rng(seed)
    means = np.stack([rng.uniform(-1, 1, P), rng.uniform(-1, 1, P), rng.uniform(2, 6, P)], 1).astype(np.float32)
    scales = np.exp(rng.normal(-4, 0.5, (P, 3))).astype(np.float32)
    rots = random_unit_quats(rng, P)
    opac = _sigmoid(rng.normal(0, 1, (P, 1))).astype(np.float32)
    sh = _sh(rng, P, degree)
    cam = identity_camera(W, H, fx=300.0 * W / 256, fy=300.0 * H / 256)
    return dict(means3D=means, scales=scales, rotations=rots, opacities=opac, shs=sh, sh_degree=degree), cam


def urban_scene(P=2_000_000, seed=1001, half_extent=500.0, buildings=400, ground_frac=0.7, degree=3):
    """Aerial urban scene: ground plane (z ~ N(0, 0.2)) plus the faces of axis-aligned boxes.

    Log-scales U[ln 0.05, ln 5] per axis; the axis along the surface normal is x0.1.
    Rotation = face frame (local z = normal) times a random yaw about the normal."""
    rng = np.random.default_rng(seed)
    n_ground = int(round(P * ground_frac))
    n_box = P - n_ground
    means = np.empty((P, 3), np.float32)
    means[:n_ground, 0] = rng.uniform(-half_extent, half_extent, n_ground)
    means[:n_ground, 1] = rng.uniform(-half_extent, half_extent, n_ground)
    means[:n_ground, 2] = rng.normal(0, 0.2, n_ground)
    # face frames: quaternion rotating local z to the normal
    s2 = math.sqrt(0.5)
    face_q = np.array([[1, 0, 0, 0],            # +z (ground / roof)
                       [s2, 0, s2, 0],          # +x
                       [s2, 0, -s2, 0],         # -x
                       [s2, -s2, 0, 0],         # +y
                       [s2, s2, 0, 0]],         # -y
                      np.float64)
    face = np.zeros(P, np.int64)
    # boxes
    bc = rng.uniform(-half_extent, half_extent, (buildings, 2))
    bs = rng.uniform(10, 60, (buildings, 2))
    bh = rng.uniform(10, 120, buildings)
    # face areas: 4 sides + roof
    areas = np.stack([bs[:, 0] * bs[:, 1], bs[:, 1] * bh, bs[:, 1] * bh, bs[:, 0] * bh, bs[:, 0] * bh], 1)
    flat = areas.reshape(-1) / areas.sum()
    pick = rng.choice(flat.size, n_box, p=flat)
    b, f = pick // 5, pick % 5
    u, v = rng.uniform(-0.5, 0.5, n_box), rng.uniform(0, 1, n_box)
    cx, cy, sx, sy, h = bc[b, 0], bc[b, 1], bs[b, 0], bs[b, 1], bh[b]
    bm = np.empty((n_box, 3))
    roof = f == 0
    bm[roof, 0] = cx[roof] + u[roof] * sx[roof]
    bm[roof, 1] = cy[roof] + (v[roof] - 0.5) * sy[roof]
    bm[roof, 2] = h[roof]
    for fi, (ax, sign) in zip((1, 2, 3, 4), ((0, 1), (0, -1), (1, 1), (1, -1))):
        m = f == fi
        if ax == 0:
            bm[m, 0] = cx[m] + sign * sx[m] / 2
            bm[m, 1] = cy[m] + u[m] * sy[m]
        else:
            bm[m, 1] = cy[m] + sign * sy[m] / 2
            bm[m, 0] = cx[m] + u[m] * sx[m]
        bm[m, 2] = v[m] * h[m]
    means[n_ground:] = bm
    face[n_ground:] = f
    lscale = rng.uniform(math.log(0.05), math.log(5.0), (P, 3))
    lscale[:, 2] += math.log(0.1)  # local z is the surface normal
    yaw = rng.uniform(0, 2 * math.pi, P)
    qy = np.stack([np.cos(yaw / 2), np.zeros(P), np.zeros(P), np.sin(yaw / 2)], 1)
    rots = quat_mul(face_q[face], qy).astype(np.float32)
    opac = _sigmoid(rng.normal(1, 1, (P, 1))).astype(np.float32)
    sh = _sh(rng, P, degree)
    return dict(means3D=means, scales=np.exp(lscale).astype(np.float32), rotations=rots, opacities=opac, shs=sh,
                sh_degree=degree)


def urban_cameras(n, seed=1003, resolutions=((640, 360), (1280, 720), (1600, 900), (1920, 1080))):
    """Batched-view cameras: resolution uniform from the set, altitude U(80,300), pitch U(30,75) deg."""
    rng = np.random.default_rng(seed)
    cams = []
    for _ in range(n):
        W, H = resolutions[rng.integers(len(resolutions))]
        cams.append(aerial_camera(rng, W=W, H=H, fx=1600.0 * W / 1920, altitude=rng.uniform(80, 300),
                                  pitch_deg=rng.uniform(30, 75)))
    return cams


def lod_tree(P=8_000_000, seed=1002, roots=2, max_branch=8, max_depth=11, half_extent=150.0, center=(0.0, 0.0)):
    """Gaussian LoD tree in BFS order.

    Branching min(Poisson(3)+1, 8); child mean = parent + N(0, parent scale); child scale = parent x 0.5;
    root log-scale U[ln 20, ln 80]; the last level is truncated at P nodes.  Returns a dict with
    xyz, log scales, raw rotations, raw opacity, SH DC + rest (degree 1), and the tree arrays
    parent [P] i32, level [P] i32, node_index [P] i32 (-1 = leaf), tree [num_internal, max_branch] i32
    (child ids, -1 padded), ancestor_path [P, max_depth+1] i32 (apps/ancestor.py layout)."""
    rng = np.random.default_rng(seed)
    parent = [np.full(roots, -1, np.int64)]
    level_nodes = [roots]
    total = roots
    counts = []
    depth = 0
    while total < P and depth < max_depth:
        nprev = level_nodes[-1]
        c = np.minimum(rng.poisson(3, nprev) + 1, max_branch)
        csum = int(c.sum())
        if total + csum > P:
            # truncate: keep children in BFS order until P is reached
            keep = P - total
            cum = np.cumsum(c)
            c = np.clip(keep - (cum - c), 0, c)
            csum = int(c.sum())
        counts.append(c)
        first = total - nprev
        parent.append(np.repeat(np.arange(first, first + nprev), c))
        level_nodes.append(csum)
        total += csum
        depth += 1
        if csum == 0:
            break
    N = total
    par = np.concatenate(parent).astype(np.int32)
    level = np.concatenate([np.full(k, d, np.int32) for d, k in enumerate(level_nodes)])
    xyz = np.empty((N, 3), np.float64)
    lsc = np.empty((N, 3), np.float64)
    xyz[:roots, 0] = rng.uniform(center[0] - half_extent, center[0] + half_extent, roots)
    xyz[:roots, 1] = rng.uniform(center[1] - half_extent, center[1] + half_extent, roots)
    xyz[:roots, 2] = rng.uniform(0, 20, roots)
    lsc[:roots] = rng.uniform(math.log(20), math.log(80), (roots, 1))
    off = roots
    for d in range(1, len(level_nodes)):
        k = level_nodes[d]
        p = par[off:off + k]
        sc = np.exp(lsc[p])
        xyz[off:off + k] = xyz[p] + rng.standard_normal((k, 3)) * sc
        lsc[off:off + k] = lsc[p] + math.log(0.5)
        off += k
    node_index = np.full(N, -1, np.int32)
    has_child = np.zeros(N, bool)
    has_child[par[par >= 0]] = True
    internal = np.nonzero(has_child)[0]
    node_index[internal] = np.arange(internal.size, dtype=np.int32)
    tree = np.full((internal.size, max_branch), -1, np.int32)
    child_ids = np.nonzero(par >= 0)[0]
    slot = np.zeros(N, np.int64)
    # child slot = rank among siblings (children are contiguous in BFS order)
    first_child = np.full(N, -1, np.int64)
    pc = par[child_ids]
    starts = np.r_[True, pc[1:] != pc[:-1]]
    first_idx = child_ids[starts]
    first_child[pc[starts]] = first_idx
    slot[child_ids] = child_ids - first_child[pc]
    tree[node_index[pc], slot[child_ids]] = child_ids
    L = len(level_nodes)
    anc = np.full((N, L), -1, np.int32)
    off = roots
    for d in range(1, L):
        k = level_nodes[d]
        ids = np.arange(off, off + k)
        p = par[ids]
        anc[ids] = anc[p]
        anc[ids, d - 1] = p
        off += k
    rots = rng.standard_normal((N, 4)).astype(np.float32)
    opac_raw = rng.normal(1, 1, (N, 1)).astype(np.float32)
    dc = rng.normal(0, 0.5, (N, 3)).astype(np.float32)
    rest = rng.normal(0, 0.1, (N, 3, 3)).astype(np.float32)
    return dict(xyz=xyz.astype(np.float32), log_scales=lsc.astype(np.float32), rotations=rots, opacity_raw=opac_raw,
                features_dc=dc, shs_rest=rest, parent=par, level=level, node_index=node_index, tree=tree,
                ancestor_path=anc, roots=np.arange(roots, dtype=np.int32))
