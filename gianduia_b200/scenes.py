"""Synthetic scene generators for the benchmark and test workloads.

Each generator writes a scene in the reference's XML format plus the OBJ meshes it
references, so that the GPU integrators and the CPU oracle consume the same files.
All randomness is seeded; the same arguments always produce the same bytes.

Workloads (sizes as named by the benchmark configurations):
  cornell      -- Cornell box, 256x256, 16 spp, path, max depth 8
  traversal    -- 1M random triangles + 16M random rays (arrays, no XML)
  microfacet   -- 1024x1024, 64 spp, path depth 16: ground quad plus a 64x64 grid of
                  displaced icospheres (1280 triangles each) with plastic / rough
                  conductor / rough glass, lit by 8 spherical emitters
  volumetric   -- the Cornell box at 512x512, 64 spp, volpath depth 32, filled with a
                  homogeneous medium (index-material boundary) plus a glass sphere
                  holding a second medium
"""
import os
import struct

import numpy as np

# ------------------------------------------------------------------ OBJ writers


def _fmt(x):
    return "%.9g" % float(x)


def write_plane_obj(path):
    """Unit quad [-0.5, 0.5]^2 in the xz plane, normal +y, with texture coordinates."""
    with open(path, "w") as f:
        f.write("v -0.5 0 -0.5\nv 0.5 0 -0.5\nv 0.5 0 0.5\nv -0.5 0 0.5\n")
        f.write("vt 0 1\nvt 1 1\nvt 1 0\nvt 0 0\n")
        f.write("vn 0 1 0\n")
        f.write("f 1/1/1 4/4/1 3/3/1\nf 1/1/1 3/3/1 2/2/1\n")


def write_cube_obj(path):
    """Unit cube [-0.5, 0.5]^3, 12 triangles, flat outward normals, per-face uvs."""
    corners = np.array([[x, y, z] for z in (-0.5, 0.5) for y in (-0.5, 0.5) for x in (-0.5, 0.5)])
    faces = [  # (corner indices counter-clockwise seen from outside, normal)
        ((0, 2, 3, 1), (0, 0, -1)), ((4, 5, 7, 6), (0, 0, 1)),
        ((0, 4, 6, 2), (-1, 0, 0)), ((1, 3, 7, 5), (1, 0, 0)),
        ((0, 1, 5, 4), (0, -1, 0)), ((2, 6, 7, 3), (0, 1, 0)),
    ]
    with open(path, "w") as f:
        for c in corners:
            f.write("v %s %s %s\n" % tuple(_fmt(v) for v in c))
        f.write("vt 0 0\nvt 1 0\nvt 1 1\nvt 0 1\n")
        for _, n in faces:
            f.write("vn %d %d %d\n" % n)
        for k, (q, _) in enumerate(faces):
            a, b, c, d = (i + 1 for i in q)
            n = k + 1
            f.write("f %d/1/%d %d/2/%d %d/3/%d\n" % (a, n, b, n, c, n))
            f.write("f %d/1/%d %d/3/%d %d/4/%d\n" % (a, n, c, n, d, n))


def write_mesh_obj(path, verts, faces, normals=None):
    """Indexed triangle mesh; per-vertex normals when given."""
    lines = ["v %s %s %s" % (_fmt(v[0]), _fmt(v[1]), _fmt(v[2])) for v in verts]
    if normals is not None:
        lines += ["vn %s %s %s" % (_fmt(n[0]), _fmt(n[1]), _fmt(n[2])) for n in normals]
        lines += ["f %d//%d %d//%d %d//%d" % (a + 1, a + 1, b + 1, b + 1, c + 1, c + 1) for a, b, c in faces]
    else:
        lines += ["f %d %d %d" % (a + 1, b + 1, c + 1) for a, b, c in faces]
    with open(path, "w") as f:
        f.write("\n".join(lines) + "\n")


# ------------------------------------------------------------------ XML helpers


def _transform(steps, name="toWorld"):
    """steps: list of ("scale", (x,y,z)) / ("rotate", (axis, angle)) / ("translate", (x,y,z))."""
    out = ['<transform name="%s">' % name]
    for kind, v in steps:
        if kind == "scale":
            out.append('<scale x="%s" y="%s" z="%s"/>' % tuple(_fmt(a) for a in v))
        elif kind == "rotate":
            axis, ang = v
            out.append('<rotate axis="%s %s %s" angle="%s"/>' % (*(_fmt(a) for a in axis), _fmt(ang)))
        elif kind == "translate":
            out.append('<translate x="%s" y="%s" z="%s"/>' % tuple(_fmt(a) for a in v))
    out.append("</transform>")
    return "\n".join(out)


def _color(name, c):
    return '<color name="%s" value="%s %s %s"/>' % (name, _fmt(c[0]), _fmt(c[1]), _fmt(c[2]))


def _filter(spec):
    """The camera's <filter> element: "box" (radius 0.5); "default": none, so the film takes
    the reference's default Gaussian filter (film.cpp:29; radius 2, alpha 2); "gaussian", or
    ("gaussian", (rx, ry), alpha), an explicit Gaussian filter (filter.h:34-54)."""
    if spec == "box":
        return ['<filter type="box"/>']
    if spec == "default":
        return []
    if spec == "gaussian":
        return ['<filter type="gaussian"/>']
    kind, radius, alpha = spec
    assert kind == "gaussian"
    return ['<filter type="gaussian">', '<vector2 name="radius" value="%s, %s"/>' % (_fmt(radius[0]), _fmt(radius[1])),
            '<float name="alpha" value="%s"/>' % _fmt(alpha), "</filter>"]


def _camera(origin, target, fov, w, h, up=(0, 1, 0), lens=None, end=None, filter="box"):
    """A pinhole camera, or with `lens` (a dict of thin-lens properties: lens_radius,
    focal_distance, k1, ca_axial, ca_lateral, vignetting, blades) a thin-lens one. `end`:
    (origin, target) of a toWorldEnd lookat (camera motion over the shutter). `filter`: see
    _filter."""
    props = []
    for k, v in sorted((lens or {}).items()):
        if isinstance(v, bool):
            props.append('<boolean name="%s" value="%s"/>' % (k, "true" if v else "false"))
        elif isinstance(v, int):
            props.append('<integer name="%s" value="%d"/>' % (k, v))
        else:
            props.append('<float name="%s" value="%s"/>' % (k, _fmt(v)))
    return "\n".join([
        '<camera type="%s">' % ("thinlens" if lens is not None else "perspective"),
        '<transform name="toWorld"><lookat origin="%s, %s, %s" target="%s, %s, %s" up="%s, %s, %s"/></transform>'
        % tuple(_fmt(v) for v in (*origin, *target, *up)),
        *([] if end is None else [
            '<transform name="toWorldEnd"><lookat origin="%s, %s, %s" target="%s, %s, %s" up="%s, %s, %s"/></transform>'
            % tuple(_fmt(v) for v in (*end[0], *end[1], *up))]),
        '<float name="fov" value="%s"/>' % _fmt(fov),
        '<integer name="width" value="%d"/>' % w,
        '<integer name="height" value="%d"/>' % h,
        *props,
        *_filter(filter),
        "</camera>",
    ])


def _medium(name, sigma_a, sigma_s, g):
    return "\n".join([
        '<medium type="homogeneous" name="%s">' % name,
        _color("sigma_a", sigma_a), _color("sigma_s", sigma_s),
        '<float name="g" value="%s"/>' % _fmt(g),
        "</medium>",
    ])


# ------------------------------------------------------------------ Cornell box


def _cornell_body(light_y=0.998):
    gray, red, green = (0.75, 0.75, 0.75), (0.63, 0.065, 0.05), (0.14, 0.45, 0.09)
    walls = [
        ([("scale", (2, 1, 2)), ("translate", (0, -1, 0))], gray),                               # floor
        ([("scale", (2, 1, 2)), ("rotate", ((1, 0, 0), 180)), ("translate", (0, 1, 0))], gray),  # ceiling
        ([("scale", (2, 1, 2)), ("rotate", ((1, 0, 0), 90)), ("translate", (0, 0, -1))], gray),  # back
        ([("scale", (2, 1, 2)), ("rotate", ((0, 0, 1), -90)), ("translate", (-1, 0, 0))], red),  # left
        ([("scale", (2, 1, 2)), ("rotate", ((0, 0, 1), 90)), ("translate", (1, 0, 0))], green),  # right
    ]
    out = []
    for k, (tr, alb) in enumerate(walls):
        shape = '<shape type="mesh" id="plane"><string name="filename" value="plane.obj"/></shape>' if k == 0 else '<ref id="plane"/>'
        out += ["<primitive>", _transform(tr), shape, '<material type="matte">', _color("albedo", alb), "</material>", "</primitive>"]
    boxes = [
        ([("scale", (0.6, 0.6, 0.6)), ("rotate", ((0, 1, 0), 18)), ("translate", (0.35, -0.7, 0.3))]),
        ([("scale", (0.6, 1.2, 0.6)), ("rotate", ((0, 1, 0), -15)), ("translate", (-0.35, -0.4, -0.3))]),
    ]
    for k, tr in enumerate(boxes):
        shape = '<shape type="mesh" id="cube"><string name="filename" value="cube.obj"/></shape>' if k == 0 else '<ref id="cube"/>'
        out += ["<primitive>", _transform(tr), shape, '<material type="matte">', _color("albedo", gray), "</material>", "</primitive>"]
    out += [
        "<primitive>",
        _transform([("scale", (0.5, 1, 0.4)), ("rotate", ((1, 0, 0), 180)), ("translate", (0, light_y, 0))]),
        '<ref id="plane"/>',
        '<material type="matte">', _color("albedo", (0, 0, 0)), "</material>",
        '<emitter type="area">', _color("radiance", (17, 12, 4)), "</emitter>",
        "</primitive>",
    ]
    return out


def cornell(out_dir, width=256, height=256, spp=16, max_depth=8, integrator="path_gpu", lens=None, filter="box"):
    """Writes the Cornell-box scene; returns the XML path. `lens`: thin-lens camera
    properties (see _camera), else a pinhole camera. `filter`: see _filter."""
    os.makedirs(out_dir, exist_ok=True)
    write_plane_obj(os.path.join(out_dir, "plane.obj"))
    write_cube_obj(os.path.join(out_dir, "cube.obj"))
    xml = ["<scene>", _camera((0, 0, 3.5), (0, 0, 0), 40, width, height, lens=lens, filter=filter),
           '<sampler type="independent"><integer name="spp" value="%d"/></sampler>' % spp,
           '<integrator type="%s"><integer name="maxDepth" value="%d"/></integrator>' % (integrator, max_depth)]
    xml += _cornell_body()
    xml.append("</scene>")
    path = os.path.join(out_dir, "cornell.xml")
    with open(path, "w") as f:
        f.write("\n".join(xml) + "\n")
    return path


def volumetric(out_dir, width=512, height=512, spp=64, max_depth=32, integrator="volpath_gpu", filter="box"):
    """Cornell box filled with a homogeneous medium plus a glass sphere with its own
    interior medium; returns the XML path. `filter`: see _filter."""
    os.makedirs(out_dir, exist_ok=True)
    write_plane_obj(os.path.join(out_dir, "plane.obj"))
    write_cube_obj(os.path.join(out_dir, "cube.obj"))
    box_med = ((0.05, 0.05, 0.05), (0.5, 0.5, 0.5), 0.6)
    xml = ["<scene>", _camera((0, 0, 3.5), (0, 0, 0), 40, width, height, filter=filter),
           '<sampler type="independent"><integer name="spp" value="%d"/></sampler>' % spp,
           '<integrator type="%s"><integer name="maxDepth" value="%d"/></integrator>' % (integrator, max_depth)]
    xml += _cornell_body(light_y=0.99)
    # medium boundary: a box inset to +-0.995, index material (null BSDF)
    xml += ["<primitive>", _transform([("scale", (1.99, 1.99, 1.99))]), '<ref id="cube"/>',
            '<material type="index">', _medium("inside", *box_med), "</material>", "</primitive>"]
    # glass sphere resting on the short box, interior medium, outside = box medium
    xml += ["<primitive>", _transform([("translate", (0.35, -0.05, 0.3))]),
            '<shape type="sphere"><float name="radius" value="0.35"/></shape>',
            '<material type="glass"><float name="eta" value="1.5"/><float name="roughness" value="0"/>',
            _medium("inside", (0.1, 0.1, 0.1), (2.0, 2.0, 2.0), -0.3),
            _medium("outside", *box_med),
            "</material>", "</primitive>"]
    xml.append("</scene>")
    path = os.path.join(out_dir, "volumetric.xml")
    with open(path, "w") as f:
        f.write("\n".join(xml) + "\n")
    return path


# ------------------------------------------------------------------ microfacet grid


def icosphere(subdiv=3):
    """Unit icosphere: icosahedron with each triangle split in four `subdiv` times
    (20 * 4^subdiv triangles; 1280 and 642 vertices for subdiv 3)."""
    t = (1.0 + 5 ** 0.5) / 2.0
    v = [(-1, t, 0), (1, t, 0), (-1, -t, 0), (1, -t, 0), (0, -1, t), (0, 1, t), (0, -1, -t), (0, 1, -t),
         (t, 0, -1), (t, 0, 1), (-t, 0, -1), (-t, 0, 1)]
    f = [(0, 11, 5), (0, 5, 1), (0, 1, 7), (0, 7, 10), (0, 10, 11), (1, 5, 9), (5, 11, 4), (11, 10, 2), (10, 7, 6),
         (7, 1, 8), (3, 9, 4), (3, 4, 2), (3, 2, 6), (3, 6, 8), (3, 8, 9), (4, 9, 5), (2, 4, 11), (6, 2, 10), (8, 6, 7),
         (9, 8, 1)]
    verts = [np.array(p, np.float64) / np.linalg.norm(p) for p in v]
    faces = f
    for _ in range(subdiv):
        cache = {}

        def mid(a, b):
            key = (min(a, b), max(a, b))
            if key not in cache:
                m = verts[a] + verts[b]
                verts.append(m / np.linalg.norm(m))
                cache[key] = len(verts) - 1
            return cache[key]
        nf = []
        for a, b, c in faces:
            ab, bc, ca = mid(a, b), mid(b, c), mid(c, a)
            nf += [(a, ab, ca), (b, bc, ab), (c, ca, bc), (ab, bc, ca)]
        faces = nf
    return np.array(verts), np.array(faces, np.int64)


def value_noise(p, seed, freq=3.0):
    """Seeded lattice value noise in [-1, 1]: hashed lattice values, trilinear blend with
    smoothstep weights. p: [n, 3] world positions."""
    q = p * freq
    i0 = np.floor(q).astype(np.int64)
    fr = q - i0
    w = fr * fr * (3.0 - 2.0 * fr)

    def h(ix, iy, iz):
        x = (ix * 73856093) ^ (iy * 19349663) ^ (iz * 83492791) ^ (seed * 2654435761)
        x = (x ^ (x >> 13)) * 1274126177
        x = x ^ (x >> 16)
        return ((x & 0xFFFFFF) / float(0xFFFFFF)) * 2.0 - 1.0
    out = 0.0
    for dx in (0, 1):
        for dy in (0, 1):
            for dz in (0, 1):
                wx = w[:, 0] if dx else 1 - w[:, 0]
                wy = w[:, 1] if dy else 1 - w[:, 1]
                wz = w[:, 2] if dz else 1 - w[:, 2]
                out = out + wx * wy * wz * h(i0[:, 0] + dx, i0[:, 1] + dy, i0[:, 2] + dz)
    return out


def microfacet(out_dir, width=1024, height=1024, spp=64, max_depth=16, grid=64, seed=2, integrator="path_gpu"):
    """Ground quad (matte 0.5) and a grid x grid of displaced icospheres (1280 triangles,
    radius 0.4, spacing 1.0, radial displacement 0.05 * value noise of the world
    position), one OBJ and one primitive each; materials uniform over plastic (IOR 1.5,
    random Kd), rough conductor (Cu-like eta/k) and rough glass (IOR 1.5), GGX alpha
    uniform in [0.05, 0.5] written as roughness = sqrt(alpha); 8 spherical emitters of
    radius 0.2 and radiance 50 above the grid. Returns the XML path (files are reused
    when the directory already holds this exact scene)."""
    os.makedirs(out_dir, exist_ok=True)
    path = os.path.join(out_dir, "microfacet.xml")
    tag = "<!-- microfacet %d %d %d %d %d %d -->" % (width, height, spp, max_depth, grid, seed)
    if os.path.exists(path):
        with open(path) as f:
            if f.readline().strip() == tag:
                return path
    rng = np.random.default_rng(seed)
    write_plane_obj(os.path.join(out_dir, "plane.obj"))
    verts, faces = icosphere(3)
    mesh_dir = os.path.join(out_dir, "spheres")
    os.makedirs(mesh_dir, exist_ok=True)
    face_lines = "\n".join("f %d %d %d" % (a + 1, b + 1, c + 1) for a, b, c in faces)
    ext = (grid - 1) * 1.0
    xml = [tag, "<scene>",
           _camera((ext / 2, ext * 0.42, -ext * 0.28), (ext / 2, 0.0, ext * 0.55), 55, width, height),
           '<sampler type="independent"><integer name="spp" value="%d"/></sampler>' % spp,
           '<integrator type="%s"><integer name="maxDepth" value="%d"/></integrator>' % (integrator, max_depth),
           "<primitive>",
           _transform([("scale", (ext + 8, 1, ext + 8)), ("translate", (ext / 2, 0, ext / 2))]),
           '<shape type="mesh"><string name="filename" value="plane.obj"/></shape>',
           '<material type="matte">' + _color("albedo", (0.5, 0.5, 0.5)) + "</material>",
           "</primitive>"]
    mats = rng.integers(0, 3, grid * grid)
    alphas = rng.uniform(0.05, 0.5, grid * grid)
    kds = rng.uniform(0.1, 0.9, (grid * grid, 3))
    for k in range(grid * grid):
        gx, gz = k % grid, k // grid
        center = np.array([gx * 1.0, 0.45, gz * 1.0])
        world = verts * 0.4 + center
        disp = 0.05 * value_noise(world, seed)
        local = verts * (0.4 + disp)[:, None]
        name = "s%04d.obj" % k
        with open(os.path.join(mesh_dir, name), "w") as f:
            f.write("\n".join("v %s %s %s" % (_fmt(a), _fmt(b), _fmt(c)) for a, b, c in local))
            f.write("\n" + face_lines + "\n")
        rough = float(np.sqrt(alphas[k]))
        if mats[k] == 0:
            m = ('<material type="plastic">' + _color("Kd", kds[k]) +
                 '<float name="eta" value="1.5"/><float name="roughness" value="%s"/></material>' % _fmt(rough))
        elif mats[k] == 1:
            m = ('<material type="conductor">' + _color("eta", (0.27, 0.68, 1.22)) + _color("k", (3.61, 2.63, 2.29)) +
                 '<float name="roughness" value="%s"/></material>' % _fmt(rough))
        else:
            m = '<material type="glass"><float name="eta" value="1.5"/><float name="roughness" value="%s"/></material>' % _fmt(rough)
        xml += ["<primitive>", _transform([("translate", tuple(center))]),
                '<shape type="mesh"><string name="filename" value="spheres/%s"/></shape>' % name, m, "</primitive>"]
    lights = np.column_stack([rng.uniform(4, ext - 4, 8), rng.uniform(2.0, 3.5, 8), rng.uniform(4, ext - 4, 8)])
    for c in lights:
        xml += ["<primitive>", _transform([("translate", tuple(c))]),
                '<shape type="sphere"><float name="radius" value="0.2"/></shape>',
                '<material type="matte">' + _color("albedo", (0, 0, 0)) + "</material>",
                '<emitter type="area">' + _color("radiance", (50, 50, 50)) + "</emitter>", "</primitive>"]
    xml.append("</scene>")
    with open(path, "w") as f:
        f.write("\n".join(xml) + "\n")
    return path


def motion(out_dir, width=64, height=64, spp=4, max_depth=8, integrator="path_gpu", camera_motion=False, lens=None,
           light_motion=True):
    """The Cornell box with motion blur (animated.cpp): the small box slides, the tall box
    turns 90 degrees about y while it rises and grows, a small emissive sphere moves
    across the room (light_motion), and with camera_motion the camera pans (toWorldEnd
    transforms, shutter time [0, 1]). Returns the XML path."""
    os.makedirs(out_dir, exist_ok=True)
    write_plane_obj(os.path.join(out_dir, "plane.obj"))
    write_cube_obj(os.path.join(out_dir, "cube.obj"))
    end = ((0.3, 0.1, 3.5), (0.1, 0.0, 0.0)) if camera_motion else None
    xml = ["<scene>", _camera((0, 0, 3.5), (0, 0, 0), 40, width, height, lens=lens, end=end),
           '<sampler type="independent"><integer name="spp" value="%d"/></sampler>' % spp,
           '<integrator type="%s"><integer name="maxDepth" value="%d"/></integrator>' % (integrator, max_depth)]
    gray = (0.75, 0.75, 0.75)
    boxes = [
        ([("scale", (0.6, 0.6, 0.6)), ("rotate", ((0, 1, 0), 18)), ("translate", (0.35, -0.7, 0.3))],
         [("scale", (0.6, 0.6, 0.6)), ("rotate", ((0, 1, 0), 18)), ("translate", (0.05, -0.7, 0.45))]),
        ([("scale", (0.6, 1.2, 0.6)), ("rotate", ((0, 1, 0), -15)), ("translate", (-0.35, -0.4, -0.3))],
         [("scale", (0.7, 1.3, 0.5)), ("rotate", ((0, 1, 0), 75)), ("translate", (-0.3, -0.3, -0.3))]),
    ]
    # the Cornell body lists the walls (5 primitives), two boxes and the light: the boxes
    # are replaced by animated ones
    prims, cur = [], []
    for line in _cornell_body():
        cur.append(line)
        if line == "</primitive>":
            prims.append(cur)
            cur = []
    new_boxes = []
    for i, (a, b) in enumerate(boxes):
        shape = '<shape type="mesh" id="cube"><string name="filename" value="cube.obj"/></shape>' if i == 0 else '<ref id="cube"/>'
        new_boxes.append(["<primitive>", _transform(a), _transform(b, name="toWorldEnd"), shape,
                          '<material type="matte">', _color("albedo", gray), "</material>", "</primitive>"])
    prims = prims[:5] + new_boxes + prims[7:]
    for p_ in prims:
        xml += p_
    if light_motion:
        xml += ["<primitive>", _transform([("translate", (-0.6, 0.5, 0.4))]),
                _transform([("translate", (0.6, 0.2, 0.1))], name="toWorldEnd"),
                '<shape type="sphere"><float name="radius" value="0.08"/></shape>',
                '<material type="matte">' + _color("albedo", (0, 0, 0)) + "</material>",
                '<emitter type="area">' + _color("radiance", (40, 30, 20)) + "</emitter>", "</primitive>"]
    xml.append("</scene>")
    path = os.path.join(out_dir, "motion.xml")
    with open(path, "w") as f:
        f.write("\n".join(xml) + "\n")
    return path


# ------------------------------------------------------------------ textures


def write_png(path, img):
    """A PNG (zlib, filter 0 on every row) from a uint8 or uint16 array [h, w, c], c = 1
    (grey), 2 (grey + alpha), 3 (RGB) or 4 (RGBA)."""
    import zlib
    img = np.asarray(img)
    if img.ndim == 2:
        img = img[..., None]
    h, w, c = img.shape
    depth = 16 if img.dtype == np.uint16 else 8
    rows = img.astype(">u2" if depth == 16 else np.uint8)
    raw = b"".join(b"\0" + rows[y].tobytes() for y in range(h))
    ctype = {1: 0, 2: 4, 3: 2, 4: 6}[c]

    def chunk(t, body):
        return struct.pack(">I", len(body)) + t + body + struct.pack(">I", zlib.crc32(t + body) & 0xFFFFFFFF)

    data = b"\x89PNG\r\n\x1a\n" + chunk(b"IHDR", struct.pack(">IIBBBBB", w, h, depth, ctype, 0, 0, 0))
    data += chunk(b"IDAT", zlib.compress(raw, 6)) + chunk(b"IEND", b"")
    with open(path, "wb") as f:
        f.write(data)


def write_exr_float(path, rgb):
    """An uncompressed scanline OpenEXR file with FLOAT R, G, B channels from [h, w, 3]."""
    rgb = np.asarray(rgb, np.float32)
    h, w, _ = rgb.shape
    header = bytearray(struct.pack("<II", 20000630, 2))

    def attr(name, typ, value):
        header.extend(name.encode() + b"\0" + typ.encode() + b"\0" + struct.pack("<i", len(value)) + value)

    attr("channels", "chlist", b"".join(c + b"\0" + struct.pack("<iBBBBii", 2, 0, 0, 0, 0, 1, 1) for c in (b"B", b"G", b"R")) + b"\0")
    attr("compression", "compression", b"\0")
    box = struct.pack("<iiii", 0, 0, w - 1, h - 1)
    attr("dataWindow", "box2i", box)
    attr("displayWindow", "box2i", box)
    attr("lineOrder", "lineOrder", b"\0")
    attr("pixelAspectRatio", "float", struct.pack("<f", 1.0))
    attr("screenWindowCenter", "v2f", struct.pack("<ff", 0.0, 0.0))
    attr("screenWindowWidth", "float", struct.pack("<f", 1.0))
    header.extend(b"\0")
    line = 8 + 12 * w
    table = b"".join(struct.pack("<Q", len(header) + 8 * h + y * line) for y in range(h))
    blocks = b"".join(struct.pack("<ii", y, 12 * w) + rgb[y, :, ::-1].T.astype("<f4").tobytes() for y in range(h))
    with open(path, "wb") as f:
        f.write(bytes(header) + table + blocks)


def _texture(kind, name, props, children=()):
    out = ['<texture type="%s" name="%s">' % (kind, name)]
    for k, v in props.items():
        if isinstance(v, str):
            out.append('<string name="%s" value="%s"/>' % (k, v))
        elif isinstance(v, int):
            out.append('<integer name="%s" value="%d"/>' % (k, v))
        elif np.ndim(v) == 0:
            out.append('<float name="%s" value="%s"/>' % (k, _fmt(v)))
        elif len(v) == 2:
            out.append('<vector2 name="%s" value="%s, %s"/>' % ((k,) + tuple(_fmt(x) for x in v)))
        elif k == "axis":
            out.append('<vector name="%s" value="%s, %s, %s"/>' % ((k,) + tuple(_fmt(x) for x in v)))
        else:
            out.append(_color(k, v))
    out += list(children)
    out.append("</texture>")
    return "\n".join(out)


def textures(out_dir, width=64, height=64, spp=4, max_depth=8, integrator="path_gpu", emitter_texture=False,
             lens=None, moving=False, point_light=False, float_textures=False, maps=False, index_box=False):
    """The Cornell box with the reference's procedural and image textures on its walls and
    boxes: Perlin turbulence (floor), cellular cracks (back wall), an sRGB PNG with linear
    filtering (left wall), a float EXR with closest filtering and clamping (right wall),
    a domain-warped checkerboard (ceiling), marble and wood (boxes); emitter_texture: the
    area light's radiance is a cellular texture; lens: thin-lens properties (see _camera);
    moving: the marble box moves over the shutter; point_light: a point light inside the
    box as well; float_textures: the left wall is a rough conductor (image R, cellular eta,
    wood_float roughness) and the wood box's plastic takes perlin_float roughness and
    checkerboard_float eta; maps: a normal map (PNG) on the back wall and a bump map
    (perlin_float) on the floor; index_box (with maps): a box of `index` material (null
    BSDF) holding a homogeneous medium, with the normal map on its faces, so that volpath
    transmittance queries cross normal-mapped boundaries. Returns the XML path."""
    os.makedirs(out_dir, exist_ok=True)
    write_plane_obj(os.path.join(out_dir, "plane.obj"))
    write_cube_obj(os.path.join(out_dir, "cube.obj"))
    rng = np.random.default_rng(7)
    y, x = np.mgrid[0:24, 0:32]
    png = np.stack([(x * 8) % 256, (y * 10) % 256, ((x + y) * 5) % 256], axis=-1).astype(np.uint8)
    write_png(os.path.join(out_dir, "wall.png"), png)
    write_exr_float(os.path.join(out_dir, "wall.exr"), rng.random((12, 16, 3)) * 0.8 + 0.1)
    tex = {
        0: _texture("perlin_color", "albedo", {"value1": (0.2, 0.25, 0.3), "value2": (0.8, 0.75, 0.6), "scale": 0.35, "octaves": 5}),
        1: _texture("domainWarp_color", "albedo", {"strength": 0.4}, [
            _texture("checkerboard_color", "base", {"value1": (0.9, 0.9, 0.9), "value2": (0.2, 0.3, 0.6), "scale": (0.25, 0.25)}),
            _texture("perlin_color", "warp", {"scale": 0.5, "octaves": 3})]),
        2: _texture("cellular_color", "albedo", {"value1": (0.1, 0.1, 0.1), "value2": (0.85, 0.8, 0.7), "scale": 0.25,
                                                  "mode": "cracks", "metric": "manhattan"}),
        3: _texture("image_color", "albedo", {"filename": "wall.png", "interpolation_mode": "linear", "color_space": "sRGB",
                                               "repeat_mode": "repeat"}),
        4: _texture("image_color", "albedo", {"filename": "wall.exr", "interpolation_mode": "closest", "repeat_mode": "clamp"}),
    }
    walls = [
        [("scale", (2, 1, 2)), ("translate", (0, -1, 0))],
        [("scale", (2, 1, 2)), ("rotate", ((1, 0, 0), 180)), ("translate", (0, 1, 0))],
        [("scale", (2, 1, 2)), ("rotate", ((1, 0, 0), 90)), ("translate", (0, 0, -1))],
        [("scale", (2, 1, 2)), ("rotate", ((0, 0, 1), -90)), ("translate", (-1, 0, 0))],
        [("scale", (2, 1, 2)), ("rotate", ((0, 0, 1), 90)), ("translate", (1, 0, 0))],
    ]
    xml = ["<scene>", _camera((0, 0, 3.5), (0, 0, 0), 40, width, height, lens=lens),
           '<sampler type="independent"><integer name="spp" value="%d"/></sampler>' % spp,
           '<integrator type="%s"><integer name="maxDepth" value="%d"/></integrator>' % (integrator, max_depth)]
    if maps:
        ny, nx = np.mgrid[0:16, 0:16]
        tilt = np.stack([np.sin(nx * 0.8) * 0.4, np.cos(ny * 0.6) * 0.3, np.ones((16, 16))], axis=-1)
        tilt /= np.linalg.norm(tilt, axis=-1, keepdims=True)
        write_png(os.path.join(out_dir, "normal.png"), np.round((tilt * 0.5 + 0.5) * 255).astype(np.uint8))
    wall_maps = {
        0: _texture("perlin_float", "bump", {"scale": 0.15, "octaves": 2}) + '<float name="bump_scale" value="0.04"/>',
        2: _texture("image_normal", "normal", {"filename": "normal.png", "interpolation_mode": "linear"}),
    } if maps else {}
    for k, tr in enumerate(walls):
        shape = '<shape type="mesh" id="plane"><string name="filename" value="plane.obj"/></shape>' if k == 0 else '<ref id="plane"/>'
        if k in wall_maps:
            mat = ['<material type="matte">', tex[k], wall_maps[k], "</material>"]
        elif float_textures and k == 3:
            mat = ['<material type="conductor">', tex[k].replace('name="albedo"', 'name="R"', 1),
                   _texture("cellular_color", "eta", {"value1": (0.2, 0.4, 1.4), "value2": (1.5, 0.9, 0.3), "scale": 0.3}),
                   _color("k", (3.0, 2.5, 2.2)),
                   _texture("wood_float", "roughness", {"value1": 0.05, "value2": 0.4, "scale": 0.5, "octaves": 2}),
                   "</material>"]
        else:
            mat = ['<material type="matte">', tex[k], "</material>"]
        xml += ["<primitive>", _transform(tr), shape] + mat + ["</primitive>"]
    boxes = [
        ([("scale", (0.6, 0.6, 0.6)), ("rotate", ((0, 1, 0), 18)), ("translate", (0.35, -0.7, 0.3))],
         _texture("marble_color", "albedo", {"scale": 0.3, "octaves": 4, "vein_freq": 8.0, "turb_scale": 3.0})),
        ([("scale", (0.6, 1.2, 0.6)), ("rotate", ((0, 1, 0), -15)), ("translate", (-0.35, -0.4, -0.3))],
         _texture("wood_color", "Kd", {"scale": 0.5, "octaves": 3, "vein_freq": 20.0, "axis": (0.0, 1.0, 0.3)})),
    ]
    for k, (tr, t) in enumerate(boxes):
        shape = '<shape type="mesh" id="cube"><string name="filename" value="cube.obj"/></shape>' if k == 0 else '<ref id="cube"/>'
        mat = ('<material type="matte">' + t + "</material>") if k == 0 else \
            ('<material type="plastic">' + t + (
                _texture("perlin_float", "roughness", {"value1": 0.05, "value2": 0.5, "scale": 0.4, "octaves": 3}) +
                _texture("checkerboard_float", "eta", {"value1": 1.3, "value2": 1.7, "scale": (0.2, 0.2)})
                if float_textures else '<float name="eta" value="1.5"/><float name="roughness" value="0.3"/>') + '</material>')
        end = [_transform(tr + [("translate", (0.15, 0.1, 0.0))], name="toWorldEnd")] if moving and k == 0 else []
        xml += ["<primitive>", _transform(tr)] + end + [shape, mat, "</primitive>"]
    if index_box:
        assert maps, "the index box carries the normal map written with maps=True"
        xml += ["<primitive>", _transform([("scale", (0.7, 0.5, 0.6)), ("rotate", ((0, 1, 0), 30)),
                                           ("translate", (0.05, 0.3, 0.2))]), '<ref id="cube"/>',
                '<material type="index">', _medium("inside", (0.2, 0.3, 0.4), (1.5, 1.2, 0.9), 0.3),
                _texture("image_normal", "normal", {"filename": "normal.png", "interpolation_mode": "linear"}),
                "</material>", "</primitive>"]
    xml += ["<primitive>",
            _transform([("scale", (0.5, 1, 0.4)), ("rotate", ((1, 0, 0), 180)), ("translate", (0, 0.998, 0))]),
            '<ref id="plane"/>', '<material type="matte">', _color("albedo", (0, 0, 0)), "</material>",
            '<emitter type="area">',
            _texture("cellular_color", "radiance", {"value1": (30, 20, 8), "value2": (4, 3, 1), "scale": 0.2})
            if emitter_texture else _color("radiance", (17, 12, 4)),
            "</emitter>", "</primitive>"]
    if point_light:
        xml.append(_emitter("point", {"position": (0.3, 0.6, 0.5), "power": (6.0, 5.0, 4.0)}))
    xml.append("</scene>")
    path = os.path.join(out_dir, "textures.xml")
    with open(path, "w") as f:
        f.write("\n".join(xml) + "\n")
    return path


# ------------------------------------------------------------------ light sources


def write_env_exr(path, width=64, height=32, sun=(0.3, 0.3), sun_size=0.04, sun_radiance=60.0):
    """Latitude-longitude environment image (column u = phi / 2 pi, row v = theta / pi,
    theta measured from +z): a sky gradient with a small bright disc (the sun) centred
    at (u, v) = `sun`. Written as an uncompressed float RGB OpenEXR file (the layout of
    gnd_image_write_exr) so that scene generation needs no compiled code."""
    v, u = np.mgrid[0:height, 0:width].astype(np.float64)
    u = (u + 0.5) / width
    v = (v + 0.5) / height
    sky = np.stack([0.2 + 0.3 * (1 - v), 0.3 + 0.4 * (1 - v), 0.5 + 0.5 * (1 - v)], axis=-1)
    du = np.minimum(np.abs(u - sun[0]), 1 - np.abs(u - sun[0]))
    disc = (du ** 2 + (v - sun[1]) ** 2) < sun_size ** 2
    img = np.where(disc[..., None], sun_radiance * np.array([1.0, 0.9, 0.7]), sky).astype(np.float32)
    header = bytearray(struct.pack("<II", 20000630, 2))

    def attr(name, typ, value):
        header.extend(name.encode() + b"\0" + typ.encode() + b"\0" + struct.pack("<i", len(value)) + value)

    attr("channels", "chlist", b"".join(c + b"\0" + struct.pack("<iBBBBii", 2, 0, 0, 0, 0, 1, 1) for c in (b"B", b"G", b"R")) + b"\0")
    attr("compression", "compression", b"\0")
    box = struct.pack("<iiii", 0, 0, width - 1, height - 1)
    attr("dataWindow", "box2i", box)
    attr("displayWindow", "box2i", box)
    attr("lineOrder", "lineOrder", b"\0")
    attr("pixelAspectRatio", "float", struct.pack("<f", 1.0))
    attr("screenWindowCenter", "v2f", struct.pack("<ff", 0.0, 0.0))
    attr("screenWindowWidth", "float", struct.pack("<f", 1.0))
    header.extend(b"\0")
    line = 8 + width * 12
    table = b"".join(struct.pack("<Q", len(header) + 8 * height + y * line) for y in range(height))
    blocks = b"".join(struct.pack("<ii", y, width * 12) + img[y, :, ::-1].T.astype("<f4").tobytes() for y in range(height))
    with open(path, "wb") as f:
        f.write(bytes(header) + table + blocks)
    return img


def _emitter(kind, props):
    out = ['<emitter type="%s">' % kind]
    for k, v in props.items():
        if isinstance(v, str):
            out.append('<string name="%s" value="%s"/>' % (k, v))
        elif np.ndim(v) == 0:
            out.append('<float name="%s" value="%s"/>' % (k, _fmt(v)))
        elif k == "position":
            out.append('<point name="%s" value="%s, %s, %s"/>' % ((k,) + tuple(_fmt(x) for x in v)))
        elif k == "direction":
            out.append('<vector name="%s" value="%s, %s, %s"/>' % ((k,) + tuple(_fmt(x) for x in v)))
        else:
            out.append(_color(k, v))
    out.append("</emitter>")
    return "\n".join(out)


LIGHTS = {
    "point": ("point", {"position": (0.6, 1.6, 0.9), "power": (60.0, 55.0, 45.0)}),
    "spot": ("spot", {"position": (-0.8, 2.0, 1.0), "direction": (0.35, -1.0, -0.45), "power": (150.0, 150.0, 150.0),
                      "spot_size": 50.0, "blend": 0.3}),
    "directional": ("directional", {"direction": (-0.4, -1.0, -0.3), "irradiance": (1.5, 1.4, 1.2)}),
}


def lights(out_dir, width=64, height=64, spp=4, max_depth=8, integrator="path_gpu", emitters=("point",), env=False,
           area=False, media=False):
    """An open scene: a ground quad and three spheres (matte, plastic, glass) under the
    given light sources: names from LIGHTS (point, spot, directional), an environment map
    (env=True, write_env_exr) and/or a small area light (area=True); standalone emitters
    come after the primitives in the file. media=True fills the glass sphere with a
    homogeneous medium (for volpath). Returns the XML path."""
    os.makedirs(out_dir, exist_ok=True)
    write_plane_obj(os.path.join(out_dir, "plane.obj"))
    xml = ["<scene>", _camera((0.0, 1.2, 4.0), (0.0, 0.3, 0.0), 40, width, height),
           '<sampler type="independent"><integer name="spp" value="%d"/></sampler>' % spp,
           '<integrator type="%s"><integer name="maxDepth" value="%d"/></integrator>' % (integrator, max_depth)]
    xml += ["<primitive>", _transform([("scale", (4, 1, 4))]),
            '<shape type="mesh"><string name="filename" value="plane.obj"/></shape>',
            '<material type="matte">' + _color("albedo", (0.6, 0.6, 0.6)) + "</material>", "</primitive>"]
    spheres = [((-0.9, 0.45, 0.0), '<material type="matte">' + _color("albedo", (0.8, 0.3, 0.2)) + "</material>"),
               ((0.0, 0.45, -0.4), '<material type="plastic">' + _color("Kd", (0.2, 0.4, 0.8)) +
                '<float name="eta" value="1.5"/><float name="roughness" value="0.3"/></material>'),
               ((0.9, 0.45, 0.2), '<material type="glass"><float name="eta" value="1.5"/>' +
                (_medium("inside", (0.05, 0.05, 0.05), (0.6, 0.5, 0.4), 0.3) if media else "") + "</material>")]
    for c, m in spheres:
        xml += ["<primitive>", _transform([("translate", c)]),
                '<shape type="sphere"><float name="radius" value="0.45"/></shape>', m, "</primitive>"]
    if area:
        xml += ["<primitive>", _transform([("translate", (0.0, 2.5, 0.5))]),
                '<shape type="sphere"><float name="radius" value="0.15"/></shape>',
                '<material type="matte">' + _color("albedo", (0, 0, 0)) + "</material>",
                '<emitter type="area">' + _color("radiance", (30, 30, 30)) + "</emitter>", "</primitive>"]
    for name in emitters:
        kind, props = LIGHTS[name]
        xml.append(_emitter(kind, props))
    if env:
        write_env_exr(os.path.join(out_dir, "sky.exr"))
        xml.append(_emitter("environment", {"filename": "sky.exr", "strength": 1.0}))
    xml.append("</scene>")
    path = os.path.join(out_dir, "lights.xml")
    with open(path, "w") as f:
        f.write("\n".join(xml) + "\n")
    return path


# ------------------------------------------------------------------ traversal micro-benchmark


def random_triangles(n=1 << 20, seed=1):
    """Triangle soup: centroids uniform in [0,1]^3, vertices = centroid + N(0, 0.01^2)
    per axis. Returns float32 [n, 3, 3]."""
    rng = np.random.default_rng(seed)
    c = rng.random((n, 1, 3), dtype=np.float64)
    e = rng.normal(0.0, 0.01, size=(n, 3, 3))
    return (c + e).astype(np.float32)


def random_rays(n=1 << 24, seed=1):
    """Rays with origins uniform in [-0.5, 1.5]^3 and directions uniform on the sphere
    (z = 1 - 2u, phi = 2 pi v); tmin = 1e-4, tmax = inf. Returns float32 [n, 8]
    laid out (ox, oy, oz, tmin, dx, dy, dz, tmax)."""
    rng = np.random.default_rng(seed + 1000)
    o = rng.uniform(-0.5, 1.5, size=(n, 3))
    u = rng.random(n)
    v = rng.random(n)
    z = 1.0 - 2.0 * u
    r = np.sqrt(np.maximum(0.0, 1.0 - z * z))
    phi = 2.0 * np.pi * v
    d = np.stack([r * np.cos(phi), r * np.sin(phi), z], axis=1)
    out = np.empty((n, 8), np.float32)
    out[:, 0:3] = o
    out[:, 3] = 1e-4
    out[:, 4:7] = d
    out[:, 7] = np.inf
    return out
