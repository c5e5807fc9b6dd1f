"""Seeded amorphous specimens written in the LAMMPS ``atomic`` data format.

The reference reads specimens with ``read_position_lammps_data_file``
(``tem_io.cpp:36-1028``): a comment line, ``N atoms``, ``T atom types``,
``lo hi xlo xhi`` (and y, z), ``Masses`` with one ``type mass`` line per type,
``Atoms``, then ``id type x y z`` lines.  Blank lines are allowed between
entries, coordinates must lie inside [lo, hi], and the mass is mapped to Z by
``guessZ`` (``tem_io.cpp:1030``; 28.0855 -> Si, Z = 14).

Positions come from random sequential addition with a minimum periodic
separation (hard-sphere exclusion), done in rounds so that large specimens
build quickly: each round proposes a block of uniform candidates, drops those
within ``min_sep`` of an accepted atom, then accepts the survivors one by one
in proposal order, rejecting any within ``min_sep`` of one accepted earlier in
the same round.  Everything is driven by ``numpy.random.default_rng(seed)``,
so a (count, box, seed) triple always yields the same file.
"""
from __future__ import annotations

import numpy as np

SI_MASS = 28.0855


def amorphous_positions(n_atoms: int, box, min_sep: float = 2.2,
                        seed: int = 0, max_rounds: int = 10_000) -> np.ndarray:
    """Return ``(n_atoms, 3)`` positions in ``[0, box)`` with periodic minimum
    separation ``min_sep`` [Angstrom]."""
    from scipy.spatial import cKDTree

    box = np.asarray(box, dtype=np.float64).reshape(3)
    rng = np.random.default_rng(seed)
    accepted = np.empty((0, 3), dtype=np.float64)
    rounds = 0
    while accepted.shape[0] < n_atoms:
        rounds += 1
        if rounds > max_rounds:
            raise RuntimeError("random sequential addition did not converge")
        need = n_atoms - accepted.shape[0]
        cand = rng.random((max(64, 2 * need), 3)) * box
        if accepted.shape[0]:
            tree = cKDTree(accepted, boxsize=box)
            d, _ = tree.query(cand, k=1, distance_upper_bound=min_sep)
            cand = cand[~np.isfinite(d) | (d >= min_sep)]
        if cand.shape[0] == 0:
            continue
        ctree = cKDTree(cand, boxsize=box)
        pairs = ctree.query_pairs(min_sep, output_type="ndarray")
        keep = np.ones(cand.shape[0], dtype=bool)
        if pairs.size:
            # a candidate is rejected if an earlier *kept* candidate is close
            nbrs = [[] for _ in range(cand.shape[0])]
            for a, b in pairs:
                lo, hi = (a, b) if a < b else (b, a)
                nbrs[hi].append(lo)
            for i in range(cand.shape[0]):
                for j in nbrs[i]:
                    if keep[j]:
                        keep[i] = False
                        break
        new = cand[keep][:need]
        accepted = np.concatenate([accepted, new], axis=0)
    return accepted


def write_lammps_data(path, positions: np.ndarray, box, mass: float = SI_MASS,
                      comment: str = "amorphous specimen") -> None:
    """Write single-species positions in the grammar the reference reads."""
    box = np.asarray(box, dtype=np.float64).reshape(3)
    n = positions.shape[0]
    with open(path, "w") as f:
        f.write("# %s\n\n" % comment)
        f.write("%d atoms\n" % n)
        f.write("1 atom types\n\n")
        f.write("0 %.6f xlo xhi\n" % box[0])
        f.write("0 %.6f ylo yhi\n" % box[1])
        f.write("0 %.6f zlo zhi\n\n" % box[2])
        f.write("Masses\n\n1 %.4f\n\n" % mass)
        f.write("Atoms\n\n")
        lines = ["%d 1 %.6f %.6f %.6f\n" % (i + 1, p[0], p[1], p[2])
                 for i, p in enumerate(positions)]
        f.writelines(lines)


def read_back(positions: np.ndarray) -> np.ndarray:
    """Positions as the reference will hold them after parsing the ``%.6f``
    text (the file is the source of truth for parity)."""
    return np.array([[float("%.6f" % v) for v in p] for p in positions])


def make_specimen(path, n_atoms: int, box, seed: int, min_sep: float = 2.2):
    """Generate and write a seeded amorphous-Si specimen; returns positions
    exactly as written (rounded to the file's 6 decimals)."""
    pos = amorphous_positions(n_atoms, box, min_sep=min_sep, seed=seed)
    pos = np.round(pos, 6)
    box = np.asarray(box, dtype=np.float64)
    pos = np.minimum(pos, np.round(box, 6))  # stay inside [lo, hi] after rounding
    write_lammps_data(path, pos, box)
    return pos
