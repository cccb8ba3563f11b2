"""The reference's xyz trajectory/restart format (MSys::write_as_xyz and
MSys::read_as_xyz, src/msys.cpp:823-941; Atom::write_as_xyz, src/atom.cpp:129-134).

    <natom>
    boundary_conditions <type> <parameters>  [comment, e.g. Time elapsed: t psec]
    <symbol>  <x> <y> <z> <type or *>  <vx> <vy> <vz>     (one line per atom)

Atom lines carry 4, 5 or 8 fields (velocities only with 8), as read_as_xyz
accepts.  Boundary conditions as BoundaryConditions' stream operators
(src/bcond.cpp:233-283): ``non_periodic``, ``cubic L``, ``orthorhombic a b c``.
Positions in A, velocities in A/ps.  Numbers are written with 17 significant
digits so a file read back gives the same doubles.
"""
import numpy as np


def _bc_text(box):
    if box is None:
        return "non_periodic"
    b = np.atleast_1d(np.asarray(box, dtype=np.float64))
    if b.size == 1:
        return f"cubic {b[0]:.17g}"
    return "orthorhombic " + " ".join(f"{x:.17g}" for x in b)


def write_xyz(f, symbols, positions, velocities=None, box=None, types=None, comment=None):
    """Write one frame to an open text file or a path."""
    if isinstance(f, str):
        with open(f, "w") as fh:
            return write_xyz(fh, symbols, positions, velocities, box, types, comment)
    r = np.asarray(positions, dtype=np.float64).reshape(-1, 3)
    v = np.zeros_like(r) if velocities is None else np.asarray(velocities, dtype=np.float64).reshape(-1, 3)
    n = len(r)
    head = f"boundary_conditions {_bc_text(box)}"
    if comment:
        head += "  " + comment
    lines = [str(n), head]
    for i in range(n):
        t = types[i] if types is not None and types[i] else "*"
        lines.append(f"{symbols[i]}  {r[i, 0]:.17g} {r[i, 1]:.17g} {r[i, 2]:.17g} {t}  "
                     f"{v[i, 0]:.17g} {v[i, 1]:.17g} {v[i, 2]:.17g}")
    f.write("\n".join(lines) + "\n")


def read_xyz(f):
    """Read one frame: dict(symbols, types, positions, velocities (None when
    no atom line has them), bctype, box, comment)."""
    if isinstance(f, str):
        with open(f) as fh:
            return read_xyz(fh)
    first = f.readline()
    if not first.endswith("\n"):
        raise ValueError("xyz: error reading line 1")
    n = int(first.split()[0])
    second = f.readline()
    if not second.endswith("\n"):
        raise ValueError("xyz: error reading line 2")
    bctype, box, comment = None, None, second.strip()
    k = second.find("boundary_conditions")
    if k >= 0:
        words = second[k + len("boundary_conditions"):].split()
        bctype = words[0]
        npar = {"non_periodic": 0, "cubic": 1, "bcc": 1, "fcc": 1, "orthorhombic": 3, "triclinic": 6}[bctype]
        vals = [float(x) for x in words[1:1 + npar]]
        box = vals[0] if npar == 1 else (np.array(vals) if npar else None)
        comment = " ".join(words[1 + npar:])
    syms, types = [], []
    r = np.zeros((n, 3))
    v = np.zeros((n, 3))
    any_v = False
    for i in range(n):
        line = f.readline()
        if not line.endswith("\n"):
            raise ValueError(f"xyz: error reading line {i + 3}")
        w = line.split()
        if len(w) not in (4, 5, 8):
            raise ValueError(f"xyz: error reading line {i + 3}")
        syms.append(w[0])
        r[i] = [float(x) for x in w[1:4]]
        types.append(w[4] if len(w) >= 5 else "*")
        if len(w) == 8:
            v[i] = [float(x) for x in w[5:8]]
            any_v = True
    return dict(symbols=syms, types=types, positions=r, velocities=v if any_v else None, bctype=bctype, box=box,
                comment=comment)


def water_symbols(nwater):
    return ["O", "H", "H"] * nwater
