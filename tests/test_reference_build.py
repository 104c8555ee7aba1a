"""The per-configuration copies of the reference's B.h (oracle/build_reference.py).

B.cu's parameters are compile-time macros, so the reference harness is built once per configuration
against a copy of B.h whose named macros get new values.  Each copy must differ from B.h in exactly
those #define lines, keep their comments, and leave an expression-valued macro (MLP_U_STEP is
`( VOXEL_WIDTH / 2)`) replaced as a whole.  Reads the reference checkout named by PCT_REFERENCE_DIR
(or the recipe's default); skipped where there is none.
"""
import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]
sys.path.insert(0, str(ROOT / "oracle"))
import build_reference as br  # noqa: E402


def header_text():
    ref = br.reference_dir(None)
    if not (ref / br.B_H).exists():
        pytest.skip("reference checkout not present")
    return (ref / br.B_H).read_text(errors="surrogateescape")


def define_value(line):
    """The value of a #define line, without its comment."""
    return line.split("//")[0].split(None, 2)[2].strip()


@pytest.mark.parametrize("name", [n for n in br.CONFIGS if n != "builtin"])
def test_patched_header_changes_exactly_the_named_macros(name):
    text = header_text()
    values = br.CONFIGS[name]
    patched = br.patched_header(text, values)
    a, b = text.splitlines(), patched.splitlines()
    assert len(a) == len(b)
    seen = set()
    for old, new in zip(a, b):
        key = new.split()[1] if new.startswith("#define") and len(new.split()) > 2 else None
        if key in values:
            seen.add(key)
            assert define_value(new) == values[key]
            if "//" in old:  # the comment survives
                assert new[new.index("//"):] == old[old.index("//"):]
        else:
            assert new == old
    assert seen == set(values)


def test_expression_macro_is_replaced_whole():
    text = header_text()
    patched = br.patched_header(text, {"MLP_U_STEP": "0.1"})
    line = [l for l in patched.splitlines() if l.startswith("#define") and l.split()[1] == "MLP_U_STEP"]
    assert len(line) == 1
    assert define_value(line[0]) == "0.1"


def test_unknown_macro_is_an_error():
    with pytest.raises(SystemExit):
        br.patched_header("#define A 1\n", {"B": "2"})
