"""CPU restatement of the reference's MD step with rigid-water constraints —
TEST INFRASTRUCTURE ONLY (tests may import it; the product never does).

Follows MDyn::run's step (src/mdyn.cpp:142-160):
  integrate_velocities(f, dt/2)      src/msys.cpp:1275-1279  v += f dt / (2m)
  integrate_positions(dt)            src/msys.cpp:1281-1285  x += v dt
  constrain_positions(dt)            src/constraint.cpp:295-335
  forces                              (the potential: this oracle's ElecLJ)
  integrate_velocities(f, dt/2)
  constrain_velocities()             src/constraint.cpp:336-358

ConstraintGroup::constrain_positions: the constraint derivatives at the
previous positions, divided by the masses, give the displacement directions;
each iteration evaluates the constraint values and derivatives at the current
positions, solves S x = -value with S[c][c'] = deriv_c(current) .
deriv_c'(previous)/m, moves the atoms by x_c deriv_c(previous)/m and the
velocities by the same over dt, until every |value| < tol.
ConstraintGroup::constrain_velocities: one solve with the current derivatives.
The water's three constraints are taken as the distances O-H1, O-H2 and H1-H2
(the reference states the angle as an angle constraint; both describe the
same rigid triangle and span the same constraint normals, so both converge
to the same positions and velocities).  ReferenceConstraints runs the
reference's own ConstraintGroup instead (oracle/_ref/libref.so), and
tests/test_md_oracle.py checks that the two agree.
"""
import numpy as np

PAIRS = ((0, 1), (0, 2), (1, 2))


def _derivs(x):
    """(nmol, 3 constraints, 3 atoms, 3) derivatives of |x_i - x_j| and the values."""
    nmol = x.shape[0]
    g = np.zeros((nmol, 3, 3, 3))
    dist = np.zeros((nmol, 3))
    for c, (i, j) in enumerate(PAIRS):
        d = x[:, i] - x[:, j]
        r = np.linalg.norm(d, axis=1)
        u = d / r[:, None]
        g[:, c, i] = u
        g[:, c, j] = -u
        dist[:, c] = r
    return g, dist


def constrain_positions(x0, x, v, minv, lengths, dt, tol=1e-12, maxit=100):
    """x0: previous positions (nmol, 3, 3); x, v updated in place."""
    g0, _ = _derivs(x0)
    sci0 = g0 * minv[:, None, :, None]
    for _ in range(maxit):
        g, dist = _derivs(x)
        val = dist - lengths[None, :]
        if np.all(np.abs(val) < tol):
            return
        S = np.einsum("mcak,mdak->mcd", g, sci0)
        lam = np.linalg.solve(S, -val[..., None])[..., 0]
        dx = np.einsum("mc,mcak->mak", lam, sci0)
        x += dx
        if dt > 0:
            v += dx / dt
    raise RuntimeError("constrain_positions did not converge")


def constrain_velocities(x, v, minv):
    g, _ = _derivs(x)
    sci0 = g * minv[:, None, :, None]
    rhs = -np.einsum("mcak,mak->mc", g, v)
    S = np.einsum("mcak,mdak->mcd", g, sci0)
    mu = np.linalg.solve(S, rhs[..., None])[..., 0]
    v += np.einsum("mc,mcak->mak", mu, sci0)


def water_lengths(r_oh=1.0, angle_deg=109.47):
    r_hh = 2 * r_oh * np.sin(np.radians(angle_deg) / 2)
    return np.array([r_oh, r_oh, r_hh])


class RestatedConstraints:
    """The constraint solves above (three distances per water)."""

    def __init__(self, lengths):
        self.lengths = lengths

    def positions(self, x0, x, v, minv, dt):
        constrain_positions(x0, x, v, minv, self.lengths, dt)

    def velocities(self, x, v, minv):
        constrain_velocities(x, v, minv)


class ReferenceConstraints:
    """The reference's own ConstraintGroup solves (oracle/_ref/libref.so:
    src/constraint.cpp with the O-H lengths and the H-O-H angle), iterated
    to tol in the reference's constraint units."""

    def __init__(self, lib, r_oh=1.0, angle_deg=109.47, tol=1e-13):
        self.lib, self.r_oh, self.angle, self.tol = lib, r_oh, angle_deg, tol

    def positions(self, x0, x, v, minv, dt):
        r, vv = self.lib.water_constrain_positions(x0, x, v, 1.0 / minv[0], dt, self.r_oh, self.angle, self.tol)
        x[...] = r.reshape(x.shape)
        v[...] = vv.reshape(v.shape)

    def velocities(self, x, v, minv):
        v[...] = self.lib.water_constrain_velocities(x, v, 1.0 / minv[0], self.r_oh, self.angle).reshape(v.shape)


def run(evaluate, r, v, masses, dt, steps, lengths, constraints=None):
    """evaluate(r (nsite,3)) -> (forces (nsite,3), potential energy).
    masses in the reference's mass unit; constraints: the solver of the
    position and velocity constraints (default: the restatement above).
    Returns the final r, v and an array (steps, 3) of kinetic, potential and
    conserved energy."""
    nmol = len(r) // 3
    x = np.array(r, dtype=np.float64).reshape(nmol, 3, 3)
    vv = np.array(v, dtype=np.float64).reshape(nmol, 3, 3)
    m = np.asarray(masses, dtype=np.float64).reshape(nmol, 3)
    minv = 1.0 / m
    cs = constraints or RestatedConstraints(lengths)
    cs.velocities(x, vv, minv)
    f, u = evaluate(x.reshape(-1, 3))
    f = f.reshape(nmol, 3, 3)
    out = np.zeros((steps, 3))
    for s in range(steps):
        vv += 0.5 * dt * f * minv[..., None]
        x0 = x.copy()
        x += dt * vv
        cs.positions(x0, x, vv, minv, dt)
        f, u = evaluate(x.reshape(-1, 3))
        f = f.reshape(nmol, 3, 3)
        vv += 0.5 * dt * f * minv[..., None]
        cs.velocities(x, vv, minv)
        ke = 0.5 * float((m[..., None] * vv * vv).sum())
        out[s] = (ke, u, ke + u)
    return x.reshape(-1, 3), vv.reshape(-1, 3), out
