// Link shims for the reference's constraint sources -- TEST INFRASTRUCTURE
// ONLY.  src/constraint.cpp's Constraint class calls three MSys methods, which
// the harness (ref_constraint.cpp, ConstraintGroup directly) never reaches:
// they stop the program if ever called.  src/atom.cpp reads its element table
// (the file _msim_elements beside this one, found through AddToSearchPath)
// with Element's stream input, which the reference's build generates from its
// io comments; here it reads this directory's own format,
// `{ atomic_number mass covalent_radius vdw_radius }`, for the few elements
// the harness needs.
#include "msys.hpp"
#include "util.h"

void MSys::change_protonation_state(int, int) { die("msys_shim: MSys::change_protonation_state is not provided"); }
void MSys::copy_positions_to(Cartesian *) const { die("msys_shim: MSys::copy_positions_to is not provided"); }
void MSys::show_as_xyz() const { die("msys_shim: MSys::show_as_xyz is not provided"); }
ostream &operator<<(ostream &s, const Element &) { die("msys_shim: Element output is not provided"); return s; }
istream &operator>>(istream &s, Element &e)
{
  char open = 0, close = 0;
  s >> open >> e.atomic_number >> e.mass >> e.covalent_radius >> e.vdw_radius >> close;
  if (open != '{' || close != '}')
    die("msys_shim: expecting { atomic_number mass covalent_radius vdw_radius }");
  return s;
}
