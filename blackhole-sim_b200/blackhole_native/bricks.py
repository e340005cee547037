"""Coefficient bricks: the host container and the seeded synthetic torus scene.

The container mirrors ``CoefficientBrickGrid`` (python/blackhole_sim/
coefficient_bricks.py:28-93): coefficients are ``[nr][ntheta][nphi][11]`` in
C order, channels in ``COEFF_NAMES`` order (coefficient_bricks.py:21-25), with
1-D strictly increasing r / theta / phi grids; theta is nonperiodic and phi is
periodic over 2*pi anchored at ``phi[0]``.
"""

from __future__ import annotations

import math
from dataclasses import dataclass

import numpy as np

COEFF_NAMES: tuple[str, ...] = (
    "j_i", "j_q", "j_u", "j_v",
    "alpha_i", "alpha_q", "alpha_u", "alpha_v",
    "rho_v", "rho_q", "rho_u",
)

# Synthetic torus scene constants.
EMISSIVITY_FRACTIONS = (1.0, 0.2, 0.1, 0.02)   # j_I, j_Q, j_U, j_V relative to the density
ABSORPTION_RATIO = 0.1                          # alpha_c = 0.1 * j_c
ROTATIVITY_SCALES = (0.5, 0.1, 0.05)            # rho_V, rho_Q, rho_U (channel order 8, 9, 10)
LOGNORMAL_SIGMA = 0.05                          # 5 % lognormal noise on every channel
TORUS_R_MAX = 40.0


def horizon_radius(a: float) -> float:
    """Outer Kerr horizon r_+ = 1 + sqrt(1 - a^2) (kerr.py:39-42)."""
    if not math.isfinite(a) or abs(a) >= 1.0:
        raise ValueError("Kerr spin must be finite and satisfy |a| < 1 for this integrator")
    return 1.0 + math.sqrt(1.0 - a * a)


def validate_grid(name: str, grid) -> np.ndarray:
    """A brick axis as contiguous float64: 1-D, >= 2 finite, strictly increasing
    values (the reference's messages, lib.rs:112-169)."""
    g = np.ascontiguousarray(np.asarray(grid, dtype=np.float64))
    if g.ndim != 1 or g.size < 2:
        raise ValueError(f"{name} grid must contain at least 2 values")
    if not np.all(np.isfinite(g)):
        raise ValueError(f"{name} grid must contain only finite values")
    if np.any(np.diff(g) <= 0.0):
        raise ValueError(f"{name} grid must be strictly increasing")
    return g


@dataclass(frozen=True)
class BrickGrid:
    """Host-side coefficient brick: grids plus ``[nr][nt][np][11]`` coefficients."""

    r: np.ndarray
    theta: np.ndarray
    phi: np.ndarray
    coeffs: np.ndarray
    spin_a: float = 0.0
    nu_hz: float = 230.0e9          # observing frequency the coefficients were computed at

    def __post_init__(self) -> None:
        for name in ("r", "theta", "phi"):
            object.__setattr__(self, name, validate_grid(name, getattr(self, name)))
        c = np.asarray(self.coeffs)
        expected = (self.r.size, self.theta.size, self.phi.size, len(COEFF_NAMES))
        if c.shape != expected:
            raise ValueError(f"coeffs must have shape {expected}; got {c.shape}")
        if c.dtype not in (np.float16, np.float32, np.float64):
            c = c.astype(np.float64)
        object.__setattr__(self, "coeffs", np.ascontiguousarray(c))

    @property
    def shape(self) -> tuple[int, int, int, int]:
        return tuple(self.coeffs.shape)  # type: ignore[return-value]

    @property
    def cells(self) -> int:
        return int(self.r.size * self.theta.size * self.phi.size)

    @property
    def dtype_name(self) -> str:
        """coefficient_bricks.py:35: the coefficients' dtype name."""
        return self.coeffs.dtype.name

    @property
    def bytes(self) -> int:
        """coefficient_bricks.py:51-53: coefficient bytes plus the grids as the
        reference stores them (float32)."""
        return int(self.coeffs.nbytes + 4 * (self.r.size + self.theta.size + self.phi.size))

    def save_npz(self, path) -> None:
        """The file layout of CoefficientBrickGrid.save_npz (coefficient_bricks.py:57-70):
        r, theta, phi, coeffs, coeff_names, nu_hz, spin_a, dtype_name; the
        reference's load_npz reads it (it keeps grids as float32)."""
        from pathlib import Path

        Path(path).parent.mkdir(parents=True, exist_ok=True)
        np.savez_compressed(path, r=self.r, theta=self.theta, phi=self.phi, coeffs=self.coeffs,
                            coeff_names=np.array(COEFF_NAMES), nu_hz=np.array(self.nu_hz),
                            spin_a=np.array(self.spin_a), dtype_name=np.array(self.coeffs.dtype.name))

    @classmethod
    def load_npz(cls, path) -> "BrickGrid":
        """Reads this class's files and the reference's (coefficient_bricks.py:72-75);
        channel order is checked when the file names its channels."""
        with np.load(path, allow_pickle=False) as z:
            if "coeff_names" in z and tuple(str(n) for n in z["coeff_names"]) != COEFF_NAMES:
                raise ValueError(f"brick channels {tuple(z['coeff_names'])} differ from {COEFF_NAMES}")
            return cls(z["r"], z["theta"], z["phi"], z["coeffs"], float(z["spin_a"]) if "spin_a" in z else 0.0,
                       float(z["nu_hz"]) if "nu_hz" in z else 230.0e9)

    def save_hdf5(self, path) -> None:
        """The HDF5 schema of CoefficientBrickGrid.save_hdf5 (coefficient_bricks.py:77-93):
        attributes schema / nu_hz / spin_a / dtype_name, gzip+shuffle datasets
        r, theta, phi, coeffs (chunked) and coeff_names.  Needs h5py."""
        try:
            import h5py  # type: ignore
        except ImportError as exc:
            raise RuntimeError("h5py is required for HDF5 coefficient bricks") from exc
        from pathlib import Path

        p = Path(path)
        p.parent.mkdir(parents=True, exist_ok=True)
        with h5py.File(p, "w") as f:
            f.attrs["schema"] = "blackhole_sim.coefficient_bricks.v1"
            f.attrs["nu_hz"] = self.nu_hz
            f.attrs["spin_a"] = self.spin_a
            f.attrs["dtype_name"] = self.coeffs.dtype.name
            for name in ("r", "theta", "phi"):
                f.create_dataset(name, data=getattr(self, name), compression="gzip", shuffle=True)
            f.create_dataset("coeffs", data=self.coeffs, compression="gzip", shuffle=True, chunks=True)
            f.create_dataset("coeff_names", data=np.asarray(COEFF_NAMES, dtype="S"))


def estimate_brick_memory(nr: int, ntheta: int, nphi: int, dtype: str = "float32") -> dict[str, float]:
    """coefficient_bricks.py:155-160: bytes of a brick's coefficients and its
    float32 grids."""
    bytes_per = np.dtype(dtype).itemsize
    coeff_bytes = int(nr) * int(ntheta) * int(nphi) * len(COEFF_NAMES) * bytes_per
    grid_bytes = (int(nr) + int(ntheta) + int(nphi)) * 4
    total = coeff_bytes + grid_bytes
    return {"coeff_bytes": float(coeff_bytes), "grid_bytes": float(grid_bytes), "total_bytes": float(total),
            "total_mib": total / (1024.0 * 1024.0)}


def torus_grids(nr: int, ntheta: int, nphi: int, spin_a: float, dtype=np.float32):
    """r log-spaced from 1.05 r_+ to 40 M; theta uniform on the open interval
    (0, pi) at cell centres; phi uniform on [0, 2 pi) without the endpoint.

    For float32 bricks the grids are rounded to float32 values, so that a
    float32 copy of a grid is exact and every consumer sees the same knots.
    """
    rp = horizon_radius(spin_a)
    r = np.geomspace(1.05 * rp, TORUS_R_MAX, int(nr))
    theta = math.pi * (np.arange(int(ntheta), dtype=np.float64) + 0.5) / int(ntheta)
    phi = np.linspace(0.0, 2.0 * math.pi, int(nphi), endpoint=False)
    if np.dtype(dtype) == np.float32:
        r, theta, phi = (g.astype(np.float32).astype(np.float64) for g in (r, theta, phi))
    return r, theta, phi


def torus_brick(nr: int, ntheta: int, nphi: int, spin_a: float, seed: int = 0, dtype=np.float32) -> BrickGrid:
    """Seeded synthetic torus brick.

    density rho = exp(-(r - 8)^2 / 8 - 4 cos^2 theta); emissivities
    j_c = f_c rho LN, absorptions alpha_c = 0.1 j_c LN', rotativities
    rho_c = s_c rho U(0.5, 1.5) LN'', where every LN is an independent
    exp(N(0, 0.05)) factor.  The generator is ``numpy.random.default_rng(seed)``
    drawn one r-slab at a time (normal (nt, np, 11), then uniform (nt, np, 3)),
    so the brick is a pure function of (shape, spin, seed, dtype).
    """
    r, theta, phi = torus_grids(nr, ntheta, nphi, spin_a, dtype)
    nr, nt, npz = r.size, theta.size, phi.size
    out_dtype = np.dtype(dtype)
    coeffs = np.empty((nr, nt, npz, 11), dtype=out_dtype)
    rng = np.random.default_rng(int(seed))
    cos2 = np.cos(theta) ** 2
    fj = np.asarray(EMISSIVITY_FRACTIONS, dtype=np.float64)
    srot = np.asarray(ROTATIVITY_SCALES, dtype=np.float64)
    for ir in range(nr):
        dens = np.exp(-((r[ir] - 8.0) ** 2) / 8.0 - 4.0 * cos2)                 # (nt,)
        ln = np.exp(rng.normal(0.0, LOGNORMAL_SIGMA, size=(nt, npz, 11)))
        u = rng.uniform(0.5, 1.5, size=(nt, npz, 3))
        d = dens[:, None, None]
        j = d * fj * ln[..., 0:4]
        slab = np.empty((nt, npz, 11), dtype=np.float64)
        slab[..., 0:4] = j
        slab[..., 4:8] = ABSORPTION_RATIO * j * ln[..., 4:8]
        slab[..., 8:11] = d * srot * u * ln[..., 8:11]
        coeffs[ir] = slab
    return BrickGrid(r, theta, phi, coeffs, spin_a=float(spin_a))
