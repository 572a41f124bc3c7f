"""Writes a Mesh as Wavefront OBJ + MTL (geometry and materials, no texture
maps) so the same scene can be read by the reference's own loader
(checker infrastructure: the oracle pins and bench.py's reference arm).
`mesh` is anything with the hp::Scene arrays: points, normals, texcoords,
triangles (v0, v1, v2, material) and materials (the 96-byte records)."""
import os

import numpy as np


def _f(x):
    return "%.9g" % float(np.float32(x))


def write_obj(mesh, directory, name):
    mtl = os.path.join(directory, name + ".mtl")
    with open(mtl, "w") as f:
        for i, m in enumerate(mesh.materials):
            f.write("newmtl m%d\n" % i)
            for key, field in (("Ka", "ambient"), ("Kd", "diffuse"), ("Ks", "specular"),
                               ("Ke", "emission")):
                f.write("%s %s %s %s\n" % ((key,) + tuple(_f(v) for v in m[field][:3])))
            f.write("Ni %s\nd %s\nNs %s\n\n" % (_f(m["optical_density"]), _f(m["dissolve"]),
                                                 _f(m["shininess"])))
    path = os.path.join(directory, name + ".obj")
    has_n = len(mesh.normals) == len(mesh.points) and len(mesh.points) > 0
    has_t = len(mesh.texcoords) == len(mesh.points) and len(mesh.points) > 0
    with open(path, "w") as f:
        f.write("mtllib %s.mtl\n" % name)
        for p in mesh.points:
            f.write("v %s %s %s\n" % (_f(p[0]), _f(p[1]), _f(p[2])))
        if has_n:
            for n in mesh.normals:
                f.write("vn %s %s %s\n" % (_f(n[0]), _f(n[1]), _f(n[2])))
        if has_t:
            for t in mesh.texcoords:
                f.write("vt %s %s\n" % (_f(t[0]), _f(t[1])))
        cur = None
        group = 0
        for tri in mesh.triangles:
            if tri[3] != cur:
                cur = tri[3]
                f.write("o g%d\nusemtl m%d\n" % (group, cur))
                group += 1
            ids = [int(v) + 1 for v in tri[:3]]
            if has_n and has_t:
                f.write("f %d/%d/%d %d/%d/%d %d/%d/%d\n" % tuple(x for i in ids for x in (i, i, i)))
            elif has_n:
                f.write("f %d//%d %d//%d %d//%d\n" % tuple(x for i in ids for x in (i, i)))
            else:
                f.write("f %d %d %d\n" % tuple(ids))
    return path
