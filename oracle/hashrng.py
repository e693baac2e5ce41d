"""Integer-hash RNG used by the CUDA path for whitewater and crown spawning.

Test infrastructure only (see ``oracle/__init__.py``).

The hash is the one the reference's WGSL uses (``hashU``/``rnd``, ``src/js/30-wgsl-sim.js:36-37``):
Wellons' "lowbias32" integer finaliser (published in his hash-prospector project). The CUDA path seeds
it from a particle's carried id instead of its buffer slot, so spawn decisions do not depend on
particle order. With this module the oracle reproduces those decisions exactly.
"""
import numpy as np

M32 = 0xFFFFFFFF


def hash_u32(x):
    """lowbias32 on uint32 arrays or ints (``30-wgsl-sim.js:36``)."""
    x = np.asarray(x, dtype=np.uint64) & M32
    x ^= x >> 16
    x = (x * 0x7feb352d) & M32
    x ^= x >> 15
    x = (x * 0x846ca68b) & M32
    x ^= x >> 16
    return x


class Stream:
    """Vectorised per-element RNG state: rnd() advances every element (``30-wgsl-sim.js:37``)."""

    def __init__(self, seed):
        self.s = np.asarray(seed, dtype=np.uint64) & M32

    def rnd(self):
        self.s = hash_u32(self.s)
        return (self.s >> 8).astype(np.float64) / 16777216.0


def seed_ww(pid, frame):
    """Seed for a whitewater spawn of particle `pid` in sub-step `frame` (cf. ``31-wgsl-sim2.js:238``)."""
    pid = np.asarray(pid, dtype=np.uint64)
    return hash_u32((pid * 9781 + np.uint64(frame) * 6271 + 17) & M32)


def drop_diameter(pid, median, sigma):
    """Lognormal diameter of sub-grid drop `pid` (the build's own rule; the reference gives every drop the
    particle mass): Box-Muller z = sqrt(-2 ln u1)·cos(2π u2) from the first two draws of the stream seeded
    hash(pid·0x9E3779B1 + 0x632BE5AB), u1 shifted by half a step off zero, |z| clamped to 4."""
    pid = np.asarray(pid, dtype=np.uint64)
    st = Stream(hash_u32((pid * 0x9E3779B1 + 0x632BE5AB) & M32))
    u1 = st.rnd() + 0.5 / 16777216.0
    u2 = st.rnd()
    z = np.clip(np.sqrt(-2.0 * np.log(u1)) * np.cos(2.0 * np.pi * u2), -4.0, 4.0)
    return median * np.exp(sigma * z)


def seed_crown(pid, frame):
    """Seed for the crown splash of particle `pid` (cf. ``31-wgsl-sim2.js:128``)."""
    pid = np.asarray(pid, dtype=np.uint64)
    return hash_u32((pid * 2654435761 + np.uint64(frame) * 97 + 3) & M32)
