"""The C++ binding a maintainer adds to the reference tree (include/eleclj_gpu.hpp,
class ElecLJGpu : ElecLJ) compiles against the reference's own headers with the
two edits it documents -- ElecLJ's `private:` label made `protected:`
(include/eleclj.hpp:361) and electrostatic_potential_at_gridpoints made
virtual (:357) -- applied to a copy of include/eleclj.hpp in a temporary
directory, never to the reference tree.  Skipped where the reference tree is
not mounted (MMNB_REFERENCE, default /root/reference)."""
import os
import shutil
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
REFERENCE = os.environ.get("MMNB_REFERENCE", "/root/reference")
HEADER = os.path.join(REFERENCE, "include", "eleclj.hpp")

needs_reference = pytest.mark.skipif(not os.path.exists(HEADER) or shutil.which("g++") is None,
                                     reason="reference tree or g++ not available")


def edited_header(tmp_path):
    src = open(HEADER).read()
    assert src.count("\nprivate:\n") == 1
    decl = "  void electrostatic_potential_at_gridpoints(const CVec gp, DVec &p);"
    assert src.count(decl) == 1
    src = src.replace("\nprivate:\n", "\nprotected:\n").replace(decl, "  virtual" + decl[1:])
    (tmp_path / "eleclj.hpp").write_text(src)


@needs_reference
def test_elecljgpu_compiles_against_the_reference_headers(tmp_path):
    edited_header(tmp_path)
    tu = tmp_path / "elecljgpu.cpp"
    tu.write_text('#include "eleclj_gpu.hpp"\n'
                  "// every member function instantiated, the virtual overrides checked\n"
                  "Potential *make_potential() { return new ElecLJGpu; }\n"
                  "void use(ElecLJGpu &g, MSys *m, double &u, Cartesian *f, const CVec gp, DVec &p)\n"
                  "{ g.init(m); g.set_lambda(0.5); g.types_changed(); g.scale(1.01);\n"
                  "  g.add_to_energy_and_forces(u, f); g.electrostatic_potential_at_gridpoints(gp, p); }\n")
    cmd = ["g++", "-std=c++11", "-Wall", "-Werror", "-c", str(tu), "-o", str(tmp_path / "elecljgpu.o"),
           f"-I{tmp_path}", f"-I{os.path.join(REFERENCE, 'include')}", f"-I{os.path.join(ROOT, 'include')}"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr


@needs_reference
def test_without_the_documented_edits_it_does_not_compile(tmp_path):
    """The edits are needed: against the unedited header the subclass cannot
    read ElecLJ's private site arrays."""
    tu = tmp_path / "elecljgpu.cpp"
    tu.write_text('#include "eleclj_gpu.hpp"\nPotential *make_potential() { return new ElecLJGpu; }\n')
    cmd = ["g++", "-std=c++11", "-fsyntax-only", str(tu), f"-I{os.path.join(REFERENCE, 'include')}",
           f"-I{os.path.join(ROOT, 'include')}"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode != 0 and "private" in r.stderr
