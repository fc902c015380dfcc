"""Parsers of the reference's restart records (io_funcs.cc:274-393), for the tests: the gas file
(float t, then per cell 18 floats + nfreq floats), the ray file (packed records ended by slot -1)
and the treion file (per cell float + 3 bools)."""
import numpy as np

GAS_FIELDS = ["rho", "temp", "nH1", "f_H1", "f_He1", "f_H2", "f_He2", "f_He3", "gamma_H1_tot", "gamma_He1_tot",
              "mfp", "mfp_912", "heat_rate", "cool_rate", "avg_nh1", "fion", "tcross", "treion_out"]


def parse_gas(raw: bytes, n3: int, nfreq: int = 5):
    t = np.frombuffer(raw[:4], np.float32)[0]
    a = np.frombuffer(raw[4:], np.float32).reshape(n3, 18 + nfreq)
    out = {k: a[:, i] for i, k in enumerate(GAS_FIELDS)}
    out["ngam_nu"] = a[:, 18:]
    out["t"] = t
    return out


def ray_dtype(nfreq: int = 5):
    return np.dtype([("slot", "<i8"), ("active", "u1"), ("order", "<i2"), ("pixel", "<i4"), ("itheta", "<u2"),
                     ("dir", "<f4", 3), ("nphot", "<f4", nfreq), ("r", "<f4"), ("dr", "<f4"), ("x", "<f4"),
                     ("y", "<f4"), ("z", "<f4"), ("time", "<f4"), ("cell", "<i4")])


def parse_rays(raw: bytes, nfreq: int = 5):
    dt = ray_dtype(nfreq)
    n = (len(raw) - 8) // dt.itemsize
    assert len(raw) == 8 + n * dt.itemsize
    assert np.frombuffer(raw[-8:], np.int64)[0] == -1
    return np.frombuffer(raw[:-8], dt)


def parse_treion(raw: bytes, n3: int):
    dt = np.dtype([("treion", "<f4"), ("flag", "u1"), ("tcross_flag", "u1"), ("neutral_flag", "u1")])
    return np.frombuffer(raw, dt, count=n3)


def ray_multiset(r):
    """Rays as a sorted list of byte strings of every field but the slot number."""
    return sorted(r[i].tobytes()[8:] for i in range(len(r)))
