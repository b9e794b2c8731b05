"""The Python 3 generic-interface generator (lamb_b200/fortran/make_interface.py).

1. A synthetic template with every rule the generator has (letters from the
   !MAKE line with or without a colon, procedures, types, a commented-out
   declaration, "end" lines) gives exactly the expected pieces.
2. Where the reference tree is present (this container; not the GPU box), all
   of its templates are regenerated and every generic module it ships as
   src/touchup/<base>.main.auto is reproduced byte for byte."""
import glob
import os
import subprocess
import sys

import pytest

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
TOOL = os.path.join(REPO, "lamb_b200", "fortran", "make_interface.py")
REF_SRC = "/root/reference/src"

TEMPLATE = """! header comment mentioning subroutine words in a comment
!MAKE: s d
module lamb_thing_X_methods
  TYPE lamb_thing_X_type
     integer :: n
  END TYPE lamb_thing_X_type
contains
  SUBROUTINE lamb_thing_X_create (thing, error)
  END SUBROUTINE lamb_thing_X_create
  function lamb_thing_X_size (thing) result (n)
  end function lamb_thing_X_size
  subroutine lamb_thing_X_hidden (x) !ignore
  end subroutine lamb_thing_X_hidden
end module lamb_thing_X_methods
"""


def _run(template, tmp, touched=False):
    auto, touch = os.path.join(tmp, "autogen"), os.path.join(tmp, "touchup")
    os.makedirs(touch, exist_ok=True)
    base = os.path.splitext(os.path.basename(template))[0].replace("_X", "")
    if touched:
        with open(os.path.join(touch, base + ".F90"), "w") as f:
            f.write("! hand-edited\n")
    subprocess.check_call([sys.executable, TOOL, template, "--autogen", auto, "--touchup", touch],
                          stdout=subprocess.DEVNULL)
    read = lambda *p: open(os.path.join(tmp, *p)).read()
    return base, read


def test_synthetic_template(tmp_path):
    t = tmp_path / "lamb_thing_X_methods.F90"
    t.write_text(TEMPLATE)
    base, read = _run(str(t), str(tmp_path))
    assert base == "lamb_thing_methods"
    assert read("autogen", base + ".uses") == "    use lamb_thing_s_methods\n    use lamb_thing_d_methods\n"
    assert read("autogen", base + ".publics") == (
        "      PUBLIC :: lamb_thing_create\n      PUBLIC :: lamb_thing_size\n"
        "      PUBLIC :: lamb_thing_s_type\n      PUBLIC :: lamb_thing_d_type\n")
    assert read("autogen", base + ".interfaces") == (
        "\n      interface lamb_thing_create\n          module procedure&\n"
        "              lamb_thing_s_create,&\n              lamb_thing_d_create\n"
        "      end interface lamb_thing_create\n"
        "\n      interface lamb_thing_size\n          module procedure&\n"
        "              lamb_thing_s_size,&\n              lamb_thing_d_size\n"
        "      end interface lamb_thing_size\n")
    assert read("autogen", base + ".contains") == ""
    mod = read("touchup", base + ".F90")
    assert mod.startswith("module lamb_thing_methods\n") and mod.endswith("end module lamb_thing_methods\n")
    for inc in ("uses", "publics", "interfaces", "contains"):
        assert f'#include "lamb_thing_methods.{inc}"' in mod
    # a hand-edited module is kept; the generated one goes next to it
    base, read = _run(str(t), str(tmp_path / "second"), touched=True)
    assert read("touchup", base + ".F90") == "! hand-edited\n"
    assert read("touchup", base + ".main.auto") == mod


def test_template_without_letters_is_refused(tmp_path):
    t = tmp_path / "lamb_none_X_types.F90"
    t.write_text("module lamb_none_X_types\nend module\n")
    r = subprocess.run([sys.executable, TOOL, str(t), "--autogen", str(tmp_path / "a"), "--touchup",
                        str(tmp_path / "t")], capture_output=True, text=True)
    assert r.returncode != 0 and "no type instantiators" in (r.stdout + r.stderr)


@pytest.mark.skipif(not os.path.isdir(REF_SRC), reason="reference tree not present")
def test_reproduces_the_reference_generic_modules(tmp_path):
    templates = sorted(glob.glob(os.path.join(REF_SRC, "*_X_*.F90")))
    assert len(templates) >= 20
    matched = 0
    for t in templates:
        base, read = _run(t, str(tmp_path), touched=True)
        shipped = os.path.join(REF_SRC, "touchup", base + ".main.auto")
        uses = read("autogen", base + ".uses").splitlines()
        assert uses and all(u.startswith("    use " + base.split("_")[0]) for u in uses)
        if os.path.exists(shipped):
            assert read("touchup", base + ".main.auto") == open(shipped).read(), base
            matched += 1
    assert matched >= 20
