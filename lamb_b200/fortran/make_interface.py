#!/usr/bin/env python3
"""Generic-interface generator for LAMB's type-templated Fortran modules.

LAMB writes each storage module once as a template, ``<name>_X_<kind>.F90``
(``kind`` in types / methods / operations / tests / util), in which ``_X``
stands for a type letter (d = real_8, s = real_4, c, z, i, l, b, w, u).  The
build instantiates one module per letter by textual substitution
(makefiles/Makefile:167-197) and then needs, per template, one generic
module that re-exports every instantiation under the letter-free names.  The
reference's tools/makeInterface.py (Python 2: ``print x``, ``except E, e``)
writes the pieces of that generic module; this is a Python 3 implementation
of the same job, producing the same files:

  <autogen>/<base>.uses        one ``use <name>_<letter>_<kind>`` line per letter
  <autogen>/<base>.interfaces  one generic interface per procedure
  <autogen>/<base>.publics     PUBLIC lines for the generic procedures and for
                               every type instantiation
  <autogen>/<base>.contains    empty
  <touchup>/<base>.F90         the generic module that #includes the above
                               (written as <base>.main.auto when a
                               hand-edited <base>.F90 already exists there)

with <base> the template's file name without ``_X`` and without extension.

Template rules (as the reference's templates use them):
  * the letters come from the first line starting with ``!MAKE`` (optional
    colon), e.g. ``!MAKE s d c z``;
  * a procedure or type is any line ``subroutine|function|type <name>`` that
    is not an ``end`` line and carries no trailing ``!`` comment (a trailing
    comment such as ``!ignore`` hides the line from the generator);
  * ``<name>`` is case-preserved; ``_X`` in it is replaced by ``_<letter>``.

Usage: python make_interface.py TEMPLATE.F90 [--autogen DIR] [--touchup DIR]
"""
from __future__ import annotations

import argparse
import os
import re
import sys
from dataclasses import dataclass, field
from typing import List

# A declaration line: optional indentation, one of the three keywords,
# whitespace, a name; the rest of the line holds no '!' (a comment excludes
# the line).  "end type" / "end subroutine" never match: "end" is not a keyword.
_DECL = re.compile(r"^\s*(subroutine|function|type)\s+([a-z0-9_]+)[^!]*$", re.IGNORECASE)

GENERIC_MODULE = """module {base}

#include "lamb_defs.h"

#include "{base}.uses"

  implicit none

  private

  character(len=*), parameter, private :: moduleN = '{base}'


#include "{base}.publics"

#include "{base}.interfaces"


  contains

#include "{base}.contains"

end module {base}
"""


@dataclass
class Template:
    path: str
    letters: List[str] = field(default_factory=list)
    procedures: List[str] = field(default_factory=list)
    types: List[str] = field(default_factory=list)

    @property
    def stem(self) -> str:
        return os.path.splitext(os.path.basename(self.path))[0]

    @property
    def base(self) -> str:
        return self.stem.replace("_X", "")


def parse(path: str) -> Template:
    t = Template(path)
    with open(path, "r", errors="replace") as f:
        for line in f:
            if line.startswith("!MAKE") and not t.letters:
                t.letters = line[6:].split()
            m = _DECL.search(line)
            if not m:
                continue
            kw, name = m.group(1).lower(), m.group(2)
            if kw == "type":
                t.types.append(name)
            else:
                t.procedures.append(name)
    return t


def instance(name: str, letter: str) -> str:
    return name.replace("_X", "_" + letter)


def render_uses(t: Template) -> str:
    return "".join(f"    use {instance(t.stem, k)}\n" for k in t.letters)


def render_interfaces(t: Template) -> str:
    out = []
    for p in t.procedures:
        generic = p.replace("_X", "")
        names = [instance(p, k) for k in t.letters]
        body = "&\n              " + ",&\n              ".join(names)
        out.append(f"\n      interface {generic}\n          module procedure{body}\n      end interface {generic}\n")
    return "".join(out)


def render_publics(t: Template) -> str:
    lines = [f"      PUBLIC :: {p.replace('_X', '')}\n" for p in t.procedures]
    lines += [f"      PUBLIC :: {instance(ty, k)}\n" for ty in t.types for k in t.letters]
    return "".join(lines)


def render_module(t: Template) -> str:
    return GENERIC_MODULE.format(base=t.base)


def generate(path: str, autogen: str, touchup: str) -> Template:
    t = parse(path)
    if not t.letters:
        raise SystemExit(f"{path}: no type instantiators (!MAKE line) specified")
    os.makedirs(autogen, exist_ok=True)
    os.makedirs(touchup, exist_ok=True)
    pieces = {"uses": render_uses(t), "interfaces": render_interfaces(t), "publics": render_publics(t),
              "contains": ""}
    for ext, text in pieces.items():
        with open(os.path.join(autogen, f"{t.base}.{ext}"), "w") as f:
            f.write(text)
    touched = os.path.join(touchup, f"{t.base}.F90")
    target = os.path.join(touchup, f"{t.base}.main.auto") if os.path.isfile(touched) else touched
    with open(target, "w") as f:
        f.write(render_module(t))
    return t


def main(argv=None) -> int:
    ap = argparse.ArgumentParser(description=__doc__.split("\n\n")[0])
    ap.add_argument("template")
    ap.add_argument("--autogen", default="autogen")
    ap.add_argument("--touchup", default="touchup")
    a = ap.parse_args(argv)
    t = generate(a.template, a.autogen, a.touchup)
    print(f"{t.base}: letters {' '.join(t.letters)}; {len(t.procedures)} procedures, {len(t.types)} types")
    return 0


if __name__ == "__main__":
    sys.exit(main())
