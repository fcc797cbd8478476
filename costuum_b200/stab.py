"""SKIRT stored-table (.stab) files from get_table output.

The layout follows the writer in the reference's TaskManager test
(test/testTaskManager.cpp:238-298, helpers :77-119): the tag "SKIRT X\\n",
the 64-bit marker 0x010203040A0BFEFF, the number of axes, the axis names,
units and scales (8-character space-padded fields), each axis as a 64-bit
count followed by its float64 values, the number of quantities with their
names, units and scales, then the values with the first axis varying
fastest (for (a, lambda, theta): for theta, for lambda, for a: one value
per quantity), and the tag "STABEND\\n". Integers and floats are written in
the host's byte order (little endian on x86-64 and on the GPU hosts).
"""
import struct

import numpy as np

MARKER = 0x010203040A0BFEFF


def _name(s):
    b = s.encode("ascii")
    if len(b) > 8:
        raise ValueError("stab names are at most 8 characters: %r" % s)
    return b + b" " * (8 - len(b))


def write(path, axes, quantities):
    """axes: list of (name, unit, scale, values); quantities: list of
    (name, unit, scale, array) with array shape (len(axis_0), len(axis_1),
    ...), axis 0 varying fastest in the file."""
    shape = tuple(len(a[3]) for a in axes)
    with open(path, "wb") as f:
        f.write(b"SKIRT X\n")
        f.write(struct.pack("<Q", MARKER))
        f.write(struct.pack("<Q", len(axes)))
        for a in axes:
            f.write(_name(a[0]))
        for a in axes:
            f.write(_name(a[1]))
        for a in axes:
            f.write(_name(a[2]))
        for a in axes:
            v = np.ascontiguousarray(a[3], np.float64)
            f.write(struct.pack("<Q", v.size))
            f.write(v.astype("<f8").tobytes())
        f.write(struct.pack("<Q", len(quantities)))
        for q in quantities:
            f.write(_name(q[0]))
        for q in quantities:
            f.write(_name(q[1]))
        for q in quantities:
            f.write(_name(q[2]))
        data = [np.asarray(q[3], np.float64) for q in quantities]
        for d in data:
            if d.shape != shape:
                raise ValueError("quantity shape %s != axes %s" % (d.shape, shape))
        # first axis fastest: transpose to C order over reversed axes
        stacked = np.stack([d.transpose(tuple(reversed(range(len(shape)))))
                            for d in data], axis=-1)
        f.write(np.ascontiguousarray(stacked, "<f8").tobytes())
        f.write(b"STABEND\n")


def read(path):
    """(axes, quantities) as written by write()."""
    with open(path, "rb") as f:
        buf = f.read()
    if buf[:8] != b"SKIRT X\n" or buf[-8:] != b"STABEND\n":
        raise ValueError("not a stab file")
    pos = 8
    (marker,) = struct.unpack_from("<Q", buf, pos)
    if marker != MARKER:
        raise ValueError("byte order marker")
    pos += 8
    (na,) = struct.unpack_from("<Q", buf, pos)
    pos += 8
    fields = []
    for _ in range(3 * na):
        fields.append(buf[pos:pos + 8].decode("ascii").rstrip())
        pos += 8
    axes = []
    for i in range(na):
        (nv,) = struct.unpack_from("<Q", buf, pos)
        pos += 8
        v = np.frombuffer(buf, "<f8", nv, pos).copy()
        pos += 8 * nv
        axes.append((fields[i], fields[na + i], fields[2 * na + i], v))
    (nq,) = struct.unpack_from("<Q", buf, pos)
    pos += 8
    qf = []
    for _ in range(3 * nq):
        qf.append(buf[pos:pos + 8].decode("ascii").rstrip())
        pos += 8
    shape = tuple(len(a[3]) for a in axes)
    nval = int(np.prod(shape)) * nq
    vals = np.frombuffer(buf, "<f8", nval, pos).reshape(tuple(reversed(shape)) + (nq,))
    quantities = []
    for j in range(nq):
        d = vals[..., j].transpose(tuple(reversed(range(len(shape)))))
        quantities.append((qf[j], qf[nq + j], qf[2 * nq + j], d.copy()))
    return axes, quantities


def write_absorption_table(path, sizes, wavelengths, thetas, table):
    """The table of the reference's test: axes (a [m, log], lambda [m, log],
    theta [rad, lin]) and quantities Qabs [1, log], Qabspol [1, lin] from a
    get_table result [size, wavelength, theta, (Qabs, Qabspol, ...)] of one
    composition."""
    t = np.asarray(table)
    return write(path,
                 [("a", "m", "log", sizes), ("lambda", "m", "log", wavelengths),
                  ("theta", "rad", "lin", thetas)],
                 [("Qabs", "1", "log", t[:, :, :, 0]),
                  ("Qabspol", "1", "lin", t[:, :, :, 1])])
