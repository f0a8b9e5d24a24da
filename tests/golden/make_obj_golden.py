"""Writes the OBJ-import fixtures (tests/golden/obj/) and records what the reference's own
loader makes of them (tests/golden/obj_golden.npz).

The fixtures are small files of this project's own making that exercise the import rules:
triangles, quads split along either diagonal, a concave hexagon and a pentagon (ear clipping),
1-based and negative indices, v/vt/vn, v//vn and bare v corners, a degenerate face, usemtl of
every material kind (Lambertian, Kd-tinted texture with -s/-o/-clamp, mirror, glass, emitter,
an unknown name), PNG textures in several encodings (RGB, RGBA, grey+alpha, 16-bit grey,
4-bit palette, Adam7-interlaced RGB, 1-bit grey) and baseline JPEG textures (4:2:0 at an odd
size, 4:2:2, 4:4:4, grey, restart intervals; written with Pillow).  The expected scenes come from the
reference's obj_scene + flatten_scene compiled from its sources (oracle/_ref/libref_cpu.so):

    make -C oracle ref REF=/root/reference && python tests/golden/make_obj_golden.py
"""
from __future__ import annotations

import struct
import sys
import zlib
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
ROOT = HERE.parents[1]
OBJ = HERE / "obj"
sys.path.insert(0, str(ROOT / "cuda-path-tracer_b200"))
sys.path.insert(0, str(ROOT / "oracle"))

import ptb200 as pt  # noqa: E402


def png(path: Path, width: int, height: int, ctype: int, depth: int, rows, palette=None, interlace=False):
    """Minimal PNG writer: rows are lists of sample values per row (already packed for < 8 bits)."""
    def chunk(kind, data):
        return struct.pack(">I", len(data)) + kind + data + struct.pack(">I", zlib.crc32(kind + data) & 0xffffffff)
    raw = b""
    if interlace:
        passes = [(0, 0, 8, 8), (4, 0, 8, 8), (0, 4, 4, 8), (2, 0, 4, 4), (0, 2, 2, 4), (1, 0, 2, 2), (0, 1, 1, 2)]
        full = rows(None)
        for x0, y0, dx, dy in passes:
            for y in range(y0, height, dy):
                line = b"".join(full[y][x] for x in range(x0, width, dx))
                if line:
                    raw += b"\x00" + line
    else:
        for y in range(height):
            raw += bytes([y % 5]) + filtered(rows(y), y % 5, rows(y - 1) if y else None, bpp(ctype, depth))
    data = struct.pack(">IIBBBBB", width, height, depth, ctype, 0, 0, 1 if interlace else 0)
    out = b"\x89PNG\r\n\x1a\n" + chunk(b"IHDR", data)
    if palette is not None:
        out += chunk(b"PLTE", bytes(palette))
    out += chunk(b"IDAT", zlib.compress(raw, 9)) + chunk(b"IEND", b"")
    path.write_bytes(out)


def bpp(ctype, depth):
    ch = {0: 1, 2: 3, 3: 1, 4: 2, 6: 4}[ctype]
    return max(1, ch * depth // 8)


def filtered(row: bytes, kind: int, prev, n: int) -> bytes:
    """Applies PNG filter `kind` (0-4) to one row, so the decoder has to undo each of them."""
    prev = prev or bytes(len(row))
    out = bytearray(len(row))
    for i, v in enumerate(row):
        a = row[i - n] if i >= n else 0
        b = prev[i]
        c = prev[i - n] if i >= n else 0
        if kind == 0:
            p = 0
        elif kind == 1:
            p = a
        elif kind == 2:
            p = b
        elif kind == 3:
            p = (a + b) // 2
        else:
            pa, pb, pc = abs(b - c), abs(a - c), abs(a + b - 2 * c)
            p = a if pa <= pb and pa <= pc else (b if pb <= pc else c)
        out[i] = (v - p) & 255
    return bytes(out)


def write_fixtures():
    OBJ.mkdir(parents=True, exist_ok=True)
    g = np.random.default_rng(20261203)
    W, H = 13, 9
    rgb = g.integers(0, 256, (H, W, 3), dtype=np.uint8)
    png(OBJ / "rgb.png", W, H, 2, 8, lambda y: rgb[y].tobytes())
    rgba = g.integers(0, 256, (H, W, 4), dtype=np.uint8)
    png(OBJ / "rgba.png", W, H, 6, 8, lambda y: rgba[y].tobytes())
    ga = g.integers(0, 256, (H, W, 2), dtype=np.uint8)
    png(OBJ / "grey_alpha.png", W, H, 4, 8, lambda y: ga[y].tobytes())
    g16 = g.integers(0, 65536, (H, W), dtype=np.uint16)
    png(OBJ / "grey16.png", W, H, 0, 16, lambda y: g16[y].astype(">u2").tobytes())
    pal = g.integers(0, 256, 16 * 3, dtype=np.uint8)
    idx = g.integers(0, 16, (H, W), dtype=np.uint8)

    def pack4(y):
        r = idx[y]
        r = np.concatenate([r, np.zeros(len(r) % 2, np.uint8)])
        return bytes(((r[0::2] << 4) | r[1::2]).tolist())
    png(OBJ / "palette4.png", W, H, 3, 4, pack4, palette=pal.tolist())
    bits = g.integers(0, 2, (H, W), dtype=np.uint8)
    png(OBJ / "grey1.png", W, H, 0, 1, lambda y: np.packbits(bits[y]).tobytes())
    inter = g.integers(0, 256, (H, W, 3), dtype=np.uint8)
    png(OBJ / "interlaced.png", W, H, 2, 8, lambda y: [[inter[r, x].tobytes() for x in range(W)] for r in range(H)], interlace=True)
    from PIL import Image
    photo = np.zeros((29, 37, 3), np.uint8)
    yy, xx = np.mgrid[0:29, 0:37]
    photo[..., 0] = (128 + 100 * np.sin(xx / 3.0)).astype(np.uint8)
    photo[..., 1] = (128 + 90 * np.cos(yy / 4.0 + xx / 7.0)).astype(np.uint8)
    photo[..., 2] = g.integers(0, 256, (29, 37), dtype=np.uint8)
    Image.fromarray(photo).save(OBJ / "jpeg420.jpg", quality=80, subsampling=2)
    Image.fromarray(photo).save(OBJ / "jpeg422.jpg", quality=90, subsampling=1)
    Image.fromarray(photo).save(OBJ / "jpeg444.jpg", quality=60, subsampling=0, restart_marker_blocks=3)
    Image.fromarray(photo[..., 1]).save(OBJ / "jpeg_grey.jpg", quality=75)
    Image.fromarray(photo[:24, :32]).save(OBJ / "jpeg_restart.jpg", quality=95, subsampling=2, restart_marker_rows=1)
    (OBJ / "fixture.mtl").write_text("""# materials of every kind the import maps
newmtl plain
Kd 0.8 0.3 0.1
illum 2
newmtl clamped
Kd 1.5 -0.2 0.4
Ks 0.1 0.1 0.1
newmtl tex_rgb
Kd 0.9 0.8 0.7
map_Kd -s 2 3 1 -o 0.25 0.5 0 rgb.png
newmtl tex_rgba
Kd 1 1 1
map_Kd -clamp on rgba.png
newmtl tex_ga
Kd 1 0.5 1
map_Kd grey_alpha.png
newmtl tex_16
map_Kd -s 0.5 grey16.png
newmtl tex_pal
Kd 0.7 0.7 0.7
map_Kd palette4.png
newmtl tex_bits
Kd 1 1 1
map_Kd -clamp off grey1.png
newmtl tex_inter
Kd 0.6 0.6 0.6
map_Kd interlaced.png
newmtl jpg420
Kd 1 1 1
map_Kd jpeg420.jpg
newmtl jpg422
Kd 0.9 0.9 0.9
map_Kd jpeg422.jpg
newmtl jpg444
Kd 1 0.8 0.6
map_Kd jpeg444.jpg
newmtl jpggrey
Kd 1 1 1
map_Kd jpeg_grey.jpg
newmtl jpgrst
Kd 1 1 1
map_Kd -clamp on jpeg_restart.jpg
newmtl mirror
Ks 0.8 0.7 0.6
illum 5
newmtl glass
Ni 1.45
illum 7
newmtl lamp
Ke 4 3 2.5
illum 2
newmtl faded
Kd 0.2 0.4 0.6
d 0.5
Ns 20
""")
    lines = ["# import fixture", "mtllib fixture.mtl", "o parts"]
    verts, uvs, nrms = [], [], []

    def v(p):
        verts.append(p)
        lines.append("v %s" % " ".join(repr(float(x)) if g.random() < 0.5 else "%.6f" % x for x in p))
        return len(verts)
    for _ in range(6):
        uvs.append(g.uniform(-0.5, 1.5, 2))
        lines.append("vt %.5f %.5f" % tuple(uvs[-1]))
    for _ in range(6):
        n = g.normal(size=3)
        nrms.append(n)
        lines.append("vn %.6f %.6f %.6e" % tuple(n))
    mats = ["plain", "clamped", "tex_rgb", "tex_rgba", "tex_ga", "tex_16", "tex_pal", "tex_bits", "tex_inter",
            "jpg420", "jpg422", "jpg444", "jpggrey", "jpgrst", "mirror",
            "glass", "lamp", "faded", "missing_name", None]
    for k, mat in enumerate(mats):
        if mat is not None:
            lines.append(f"usemtl {mat}")
        c = g.uniform(-2, 2, 3)
        # a triangle with v/vt/vn corners, 1-based
        a, b, d = (v(c + g.normal(size=3) * 0.5) for _ in range(3))
        lines.append(f"f {a}/{1 + k % 6}/{1 + k % 6} {b}/{1 + (k + 1) % 6}/{1 + (k + 2) % 6} {d}/{1 + (k + 3) % 6}/{1 + (k + 4) % 6}")
        # a quad with negative indices and v//vn corners (either diagonal, by construction)
        q = [c + np.array([0.1, 0, 0]), c + np.array([0.9, 0.05 * k, 0.1]), c + np.array([1.0, 1.0, 0.2]),
             c + np.array([0.0, 0.7 + 0.2 * (k % 3), 0.1])]
        for p in q:
            v(p)
        lines.append(f"f -4//{1 + k % 6} -3//{1 + (k + 1) % 6} -2//{1 + (k + 2) % 6} -1//{1 + (k + 3) % 6}")
    lines.append("g polygons")
    lines.append("usemtl plain")
    # a concave hexagon in the xz plane and a pentagon in a tilted plane (bare v corners)
    hexa = [(0, 0, 0), (2, 0, 0), (2, 0, 2), (1, 0, 1), (0, 0, 2), (-0.5, 0, 1)]
    ids = [v(np.array(p) + [0, -3, 0]) for p in hexa]
    lines.append("f " + " ".join(str(i) for i in ids))
    pent = [(0, 0, 0), (1, 0.2, 0), (1.3, 0.8, 0.3), (0.5, 1.4, 0.5), (-0.3, 0.8, 0.2)]
    ids = [v(np.array(p) + [3, 0, -1]) for p in pent]
    lines.append("usemtl tex_rgb")
    lines.append("f " + " ".join(str(i) for i in ids))
    # a degenerate face (a repeated corner: zero area) is skipped
    ids = [v(np.array(p)) for p in ((5, 5, 5), (6, 6, 6))]
    lines.append("f %d %d %d" % (ids[0], ids[1], ids[0]))
    lines.append("l 1 2")
    (OBJ / "fixture.obj").write_text("\n".join(lines) + "\n")


CASES = [
    ("plain", 320, 200, (1, 1, 1), (0, 0, 0), (0, 0, 0)),
    ("tall", 120, 300, (1, 1, 1), (0, 0, 0), (0, 0, 0)),
    ("transformed", 200, 200, (1.5, 0.5, 2.0), (30, -45, 400), (0.25, -1.0, 3.0)),
    ("mirrored", 160, 90, (-1.0, 1.0, 1.0), (0, 90, 0), (0, 0, 0)),
]


def main():
    from oracle_bind import RefCpu
    write_fixtures()
    ref = RefCpu()
    out = {}
    for name, w, h, sc, rot, tr in CASES:
        scene, cam = ref.flat_obj(OBJ / "fixture.obj", w, h, sc, rot, tr)
        out.update({f"{name}_triangles": scene.triangles, f"{name}_spheres": scene.spheres, f"{name}_materials": scene.materials,
                    f"{name}_textures": scene.textures, f"{name}_pixels": scene.pixels, f"{name}_camera": cam,
                    f"{name}_args": np.array([w, h, *sc, *rot, *tr], np.float64)})
    np.savez_compressed(HERE / "obj_golden.npz", **out)
    print("wrote", HERE / "obj_golden.npz", sum(v.nbytes for v in out.values()), "bytes")


if __name__ == "__main__":
    main()
