"""The ncu summaries under profiles/ give the command that made each figure.
Every `python bench.py ...` command quoted there must still be accepted by
bench.py's option parser, so that the command can be run again as written."""
import pathlib
import re
import shlex
import sys

import pytest

ROOT = pathlib.Path(__file__).resolve().parents[1]
sys.path.insert(0, str(ROOT))


def _commands():
    out = []
    for md in sorted((ROOT / "profiles").glob("*.md")):
        # join shell continuation lines, then take what follows `python bench.py`
        text = re.sub(r"\\\n\s*", " ", md.read_text())
        for m in re.finditer(r"python bench\.py([^\n`]*)", text):
            out.append((md.name, m.group(1).strip()))
    return out


COMMANDS = _commands()


def test_profiles_quote_commands():
    assert COMMANDS, "no bench.py command found under profiles/"


@pytest.mark.parametrize("name,args", COMMANDS, ids=[f"{n}:{a}" for n, a in COMMANDS])
def test_profile_command_parses(name, args, monkeypatch):
    import bench

    monkeypatch.setattr(sys, "argv", ["bench.py"] + shlex.split(args))
    try:
        bench.parse()
    except SystemExit as e:  # argparse rejects an unknown or malformed option
        pytest.fail(f"{name}: `python bench.py {args}` is rejected by bench.py ({e})")
