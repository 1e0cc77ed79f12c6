"""Seeded synthetic volumes restated with torch tensor operations.

TEST INFRASTRUCTURE ONLY, beside the CPU oracle: the inputs of the
reference arm of bench.py (which must not load libvt.so) and a second,
independent statement of libvt's generators (csrc/gen.cu) that the tests
compare them with.  Every float operation is a separate torch kernel, so
it rounds once, in the order gen.cu writes it (compiled there without
contraction); integer hashing is splitmix64 on int64 tensors with logical
shifts.  On a CUDA device the results equal vt_generate_volume_device bit
for bit; on the CPU the blob term's exp may differ from the device's by an
ulp.

  sphere : |x - c| + sigma * g, g a 4-term Irwin-Hall normal from
           splitmix64 counters 2k, 2k+1 of voxel k
  blobs  : sum of anisotropic Gaussian blobs + 4-octave value noise
  fractal: 6-octave value noise quantised to 0..255, spheres of a constant
           value on top (uint8)
"""
import numpy as np

_M64 = (1 << 64) - 1


def _s64(v):
    """unsigned 64-bit constant as the int64 with the same bits"""
    v &= _M64
    return v - (1 << 64) if v >= 1 << 63 else v


def _srl(torch, x, k):
    """logical right shift of int64 bits"""
    return (x >> k) & ((1 << (64 - k)) - 1)


def sm64_t(torch, z):
    """splitmix64 (Steele, Lea, Flood 2014) on an int64 tensor"""
    z = z + _s64(0x9E3779B97F4A7C15)
    z = (z ^ _srl(torch, z, 30)) * _s64(0xBF58476D1CE4E5B9)
    z = (z ^ _srl(torch, z, 27)) * _s64(0x94D049BB133111EB)
    return z ^ _srl(torch, z, 31)


def sm64_int(z):
    """splitmix64 on a Python int (host-side parameter draws)"""
    z = (z + 0x9E3779B97F4A7C15) & _M64
    z = ((z ^ (z >> 30)) * 0xBF58476D1CE4E5B9) & _M64
    z = ((z ^ (z >> 27)) * 0x94D049BB133111EB) & _M64
    return z ^ (z >> 31)


def u01_int(h):
    return np.float32(h >> 40) * np.float32(5.9604644775390625e-08)


def blob_params(seed, dims, prm):
    """Blob centres, 0.5/sigma^2 per axis and amplitudes as gen.cu's
    make_blobs draws them (float32 arithmetic)."""
    f = np.float32
    nb = int(prm[0]) if len(prm) > 0 else 256
    smin, smax = (f(prm[1]), f(prm[2])) if len(prm) > 2 else (f(20.0), f(120.0))
    amin, amax = (f(prm[3]), f(prm[4])) if len(prm) > 4 else (f(0.5), f(1.5))
    noise = f(prm[5]) if len(prm) > 5 else f(0.05)
    k = sm64_int(seed ^ 0xB10B5)
    out = []
    for i in range(nb):
        u = [u01_int(sm64_int((k + i * 7 + j) & _M64)) for j in range(7)]
        cx, cy, cz = u[0] * f(dims[0]), u[1] * f(dims[1]), u[2] * f(dims[2])
        sx, sy, sz = (smin + (smax - smin) * u[3], smin + (smax - smin) * u[4], smin + (smax - smin) * u[5])
        out.append((cx, cy, cz, f(0.5) / (sx * sx), f(0.5) / (sy * sy), f(0.5) / (sz * sz),
                    amin + (amax - amin) * u[6]))
    return out, noise


def sphere_params(seed, dims, prm):
    f = np.float32
    ns = int(prm[0]) if len(prm) > 0 else 32
    rmin, rmax = (f(prm[1]), f(prm[2])) if len(prm) > 2 else (f(50.0), f(400.0))
    sval = int(prm[3]) if len(prm) > 3 else 200
    k = sm64_int(seed ^ 0x5FE4E)
    out = []
    for i in range(ns):
        u = [u01_int(sm64_int((k + i * 4 + j) & _M64)) for j in range(4)]
        r = rmin + (rmax - rmin) * u[3]
        out.append((u[0] * f(dims[0]), u[1] * f(dims[1]), u[2] * f(dims[2]), r * r))
    return out, sval


class _Lattice:
    """Lattice values of one noise octave over the lattice points a box of
    voxels needs (value_noise's lattice(), gen.cu), looked up by index."""

    def __init__(self, torch, seed, lo, hi, octave, dev):
        self.lo = lo
        n = [hi[a] - lo[a] + 2 for a in range(3)]
        ix = torch.arange(lo[0], lo[0] + n[0], dtype=torch.int64, device=dev).view(-1, 1, 1)
        iy = torch.arange(lo[1], lo[1] + n[1], dtype=torch.int64, device=dev).view(1, -1, 1)
        iz = torch.arange(lo[2], lo[2] + n[2], dtype=torch.int64, device=dev).view(1, 1, -1)
        key = ((ix * 1048583 + iy) * 1048589 + iz) * 16 + octave
        h = sm64_int((seed ^ 0x5bd1e9955bd1e995) & _M64)
        v = sm64_t(torch, key) ^ _s64(h)
        u = _srl(torch, v, 40).to(torch.float32) * 5.9604644775390625e-08
        self.v = (u * 2.0 - 1.0).contiguous()
        self.n = n

    def at(self, ix, iy, iz):
        return self.v[ix - self.lo[0], iy - self.lo[1], iz - self.lo[2]]


def _value_noise(torch, lat, x, y, z, cell):
    cell = torch.full((1, 1, 1), cell, dtype=torch.float32, device=x.device)
    fx, fy, fz = x / cell, y / cell, z / cell
    flx, fly, flz = torch.floor(fx), torch.floor(fy), torch.floor(fz)
    ix, iy, iz = flx.to(torch.int64), fly.to(torch.int64), flz.to(torch.int64)

    def smooth(t):
        return (t * t) * (3.0 - 2.0 * t)
    tx, ty, tz = smooth(fx - flx), smooth(fy - fly), smooth(fz - flz)
    v000, v001 = lat.at(ix, iy, iz), lat.at(ix, iy, iz + 1)
    v010, v011 = lat.at(ix, iy + 1, iz), lat.at(ix, iy + 1, iz + 1)
    v100, v101 = lat.at(ix + 1, iy, iz), lat.at(ix + 1, iy, iz + 1)
    v110, v111 = lat.at(ix + 1, iy + 1, iz), lat.at(ix + 1, iy + 1, iz + 1)
    a00, a01 = v000 + (v100 - v000) * tx, v001 + (v101 - v001) * tx
    a10, a11 = v010 + (v110 - v010) * tx, v011 + (v111 - v011) * tx
    b0, b1 = a00 + (a10 - a00) * ty, a01 + (a11 - a01) * ty
    return b0 + (b1 - b0) * tz


def _fractal(torch, seed, x, y, z, cell, octaves, box):
    """gen.cu's fractal(): octave sum over the voxel coordinates x, y, z
    (float32 tensors broadcast to the box) of lattice cell `cell`."""
    dev = x.device
    s = torch.zeros(torch.broadcast_shapes(x.shape, y.shape, z.shape), dtype=torch.float32, device=dev)
    amp, norm, c = np.float32(1.0), np.float32(0.0), np.float32(cell)
    for o in range(octaves):
        lo = [int(np.floor(np.float32(box[0][a]) / c)) - 1 for a in range(3)]
        hi = [int(np.floor(np.float32(box[1][a]) / c)) + 1 for a in range(3)]
        lat = _Lattice(torch, seed, lo, hi, o, dev)
        s = s + float(amp) * _value_noise(torch, lat, x, y, z, float(c))
        norm = np.float32(norm + amp)
        amp = np.float32(amp * np.float32(0.5))
        c = np.float32(c * np.float32(0.5))
    # a tensor divisor: torch turns division by a Python scalar into a
    # multiplication by its reciprocal, which rounds differently
    return s / torch.full_like(s, float(norm))


def _coords(torch, x0, x1, ny, nz, dev):
    x = torch.arange(x0, x1, dtype=torch.float32, device=dev).view(-1, 1, 1)
    y = torch.arange(0, ny, dtype=torch.float32, device=dev).view(1, -1, 1)
    z = torch.arange(0, nz, dtype=torch.float32, device=dev).view(1, 1, -1)
    return x, y, z


def generate(torch, kind, seed, dims, params, out, dev, slab=64):
    """Fills `out` (a host or device tensor of dims voxels, x slowest:
    float32 for sphere/blobs, uint8 for fractal) slab by slab, computing
    on `dev`.  kind: "sphere", "blobs" or "fractal"."""
    nx, ny, nz = (int(d) for d in dims)
    f32 = np.float32
    if kind == "blobs":
        blobs, noise = blob_params(seed, dims, params)
    elif kind == "fractal":
        sph, sval = sphere_params(seed, dims, params)
    else:
        c = [f32(p) for p in params[:3]] if len(params) >= 3 else [f32((d - 1) * 0.5) for d in dims]
        sigma = f32(params[3]) if len(params) > 3 else f32(0.25)
    for x0 in range(0, nx, slab):
        x1 = min(nx, x0 + slab)
        x, y, z = _coords(torch, x0, x1, ny, nz, dev)
        if kind == "sphere":
            dx, dy, dz = x - float(c[0]), y - float(c[1]), z - float(c[2])
            # sqrt in double, rounded once to float: the correctly rounded
            # float square root (torch's float32 CPU sqrt is not)
            r = torch.sqrt(((dx * dx + dy * dy) + dz * dz).double()).float()
            xi = torch.arange(x0, x1, dtype=torch.int64, device=dev).view(-1, 1, 1)
            yi = torch.arange(0, ny, dtype=torch.int64, device=dev).view(1, -1, 1)
            zi = torch.arange(0, nz, dtype=torch.int64, device=dev).view(1, 1, -1)
            k = (xi * ny + yi) * nz + zi
            r0 = sm64_t(torch, seed + 2 * k)
            r1 = sm64_t(torch, seed + 2 * k + 1)
            m24 = 0xFFFFFF
            S = _srl(torch, r0, 40) + (_srl(torch, r0, 16) & m24) + _srl(torch, r1, 40) + (_srl(torch, r1, 16) & m24)
            g = (S.to(torch.float32) * 5.9604644775390625e-08 - 2.0) * 1.7320508075688772
            v = r + float(sigma) * g
        elif kind == "blobs":
            v = torch.zeros((x1 - x0, ny, nz), dtype=torch.float32, device=dev)
            for (cx, cy, cz, ix2, iy2, iz2, amp) in blobs:
                # outside the box where one axis alone gives e >= 40 the blob
                # adds nothing (gen.cu skips e >= 40); a voxel of margin
                # covers the rounding of dx*dx*ix2
                hx = float(np.sqrt(40.0 / float(ix2))) + 2.0
                hy = float(np.sqrt(40.0 / float(iy2))) + 2.0
                hz = float(np.sqrt(40.0 / float(iz2))) + 2.0
                bx0, bx1 = max(x0, int(np.floor(cx - hx))), min(x1, int(np.ceil(cx + hx)) + 1)
                by0, by1 = max(0, int(np.floor(cy - hy))), min(ny, int(np.ceil(cy + hy)) + 1)
                bz0, bz1 = max(0, int(np.floor(cz - hz))), min(nz, int(np.ceil(cz + hz)) + 1)
                if bx0 >= bx1 or by0 >= by1 or bz0 >= bz1:
                    continue
                sub = v[bx0 - x0:bx1 - x0, by0:by1, bz0:bz1]
                ddx = x[bx0 - x0:bx1 - x0] - float(cx)
                ddy = y[:, by0:by1] - float(cy)
                ddz = z[:, :, bz0:bz1] - float(cz)
                e = ((ddx * ddx) * float(ix2) + (ddy * ddy) * float(iy2)) + (ddz * ddz) * float(iz2)
                add = float(amp) * torch.exp(-e)
                sub.copy_(torch.where(e < 40.0, sub + add, sub))
            fr = _fractal(torch, seed, x, y, z, 128.0, 4, ((x0, 0, 0), (x1, ny, nz)))
            v = v + float(noise) * fr
        else:
            fr = _fractal(torch, seed, x, y, z, 256.0, 6, ((x0, 0, 0), (x1, ny, nz)))
            u = 0.5 + 0.5 * fr
            u = torch.clamp(u, 0.0, 1.0)
            q = (u * 255.0 + 0.5).to(torch.uint8)
            inside = torch.zeros((x1 - x0, ny, nz), dtype=torch.bool, device=dev)
            for (cx, cy, cz, r2) in sph:
                dx, dy, dz = x - float(cx), y - float(cy), z - float(cz)
                inside |= ((dx * dx + dy * dy) + dz * dz) < float(r2)
            v = torch.where(inside, torch.full_like(q, sval), q)
        out[x0:x1].copy_(v.reshape(x1 - x0, ny, nz))
    return out
