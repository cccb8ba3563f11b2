// Harness over the reference's own constraint solver -- TEST INFRASTRUCTURE
// ONLY.  The reference's src/constraint.cpp is compiled in this translation
// unit from where it lies (its ConstraintGroup, LengthCnstr and AngleCnstr
// classes are local to that file); nothing of it is copied here.
//
// orc_water_constrain_positions / orc_water_constrain_velocities apply, to
// each rigid water [O, H, H], one ConstraintGroup holding the constraints
// Constraint::add_constraints builds for it (src/constraint.cpp:381-436): the
// two O-H bond lengths and the H-O-H angle (AngleCnstr(H1, O, H2)), solved by
// ConstraintGroup::constrain_positions / constrain_velocities
// (src/constraint.cpp:295-358) with the reference's tolerance rule and
// LinearSolve (src/linalg.cpp:29-37).
#include "constraint.cpp"

extern "C" {

// directory holding the element table src/atom.cpp reads (_msim_elements)
void orc_add_search_path(const char *dir) { AddToSearchPath(dir); }

// r0: positions before the drift, r and v: after it (updated in place), all
// 9 doubles per molecule; mass: the three site masses; dt: the step.
int orc_water_constrain_positions(int nmol, const double *r0, double *r, double *v, const double *mass, double dt,
                                  double r_oh, double angle_deg, double tol, int maxit)
{
  Element el[3];
  for (int k = 0; k < 3; k++) {
    el[k].atomic_number = k == 0 ? 8 : 1;
    el[k].mass = mass[k];
    el[k].covalent_radius = el[k].vdw_radius = 0;
  }
  for (int m = 0; m < nmol; m++) {
    Lst<Cnstr *> cl;
    cl.add(new LengthCnstr(0, 1, r_oh));
    cl.add(new LengthCnstr(0, 2, r_oh));
    cl.add(new AngleCnstr(1, 0, 2, angle_deg));
    {
      ConstraintGroup g(cl);
      Vec<Atom> at(3);
      CVec c0(3);
      for (int k = 0; k < 3; k++) {
        const double *p0 = r0 + 9 * m + 3 * k, *p = r + 9 * m + 3 * k, *w = v + 9 * m + 3 * k;
        c0[k] = Cartesian(p0[0], p0[1], p0[2]);
        at[k].position = Cartesian(p[0], p[1], p[2]);
        at[k].velocity = Cartesian(w[0], w[1], w[2]);
        at[k].element = &el[k];
      }
      g.constrain_positions(c0, at, dt, tol, maxit, 0);
      for (int k = 0; k < 3; k++) {
        double *p = r + 9 * m + 3 * k, *w = v + 9 * m + 3 * k;
        p[0] = at[k].position.x;
        p[1] = at[k].position.y;
        p[2] = at[k].position.z;
        w[0] = at[k].velocity.x;
        w[1] = at[k].velocity.y;
        w[2] = at[k].velocity.z;
      }
    }
    LstItr<Cnstr *> c;
    for (c.init(cl); c.ok(); c.next())
      delete c();
  }
  return 0;
}

// v projected onto the constraints at r (ConstraintGroup::constrain_velocities)
int orc_water_constrain_velocities(int nmol, const double *r, double *v, const double *mass, double r_oh,
                                   double angle_deg)
{
  Element el[3];
  for (int k = 0; k < 3; k++) {
    el[k].atomic_number = k == 0 ? 8 : 1;
    el[k].mass = mass[k];
    el[k].covalent_radius = el[k].vdw_radius = 0;
  }
  for (int m = 0; m < nmol; m++) {
    Lst<Cnstr *> cl;
    cl.add(new LengthCnstr(0, 1, r_oh));
    cl.add(new LengthCnstr(0, 2, r_oh));
    cl.add(new AngleCnstr(1, 0, 2, angle_deg));
    {
      ConstraintGroup g(cl);
      Vec<Atom> at(3);
      for (int k = 0; k < 3; k++) {
        const double *p = r + 9 * m + 3 * k, *w = v + 9 * m + 3 * k;
        at[k].position = Cartesian(p[0], p[1], p[2]);
        at[k].velocity = Cartesian(w[0], w[1], w[2]);
        at[k].element = &el[k];
      }
      g.constrain_velocities(at);
      for (int k = 0; k < 3; k++) {
        double *w = v + 9 * m + 3 * k;
        w[0] = at[k].velocity.x;
        w[1] = at[k].velocity.y;
        w[2] = at[k].velocity.z;
      }
    }
    LstItr<Cnstr *> c;
    for (c.init(cl); c.ok(); c.next())
      delete c();
  }
  return 0;
}

}  // extern "C"
