"""Every ncu summary under profiles/ names the bench.py command it was
captured from; those commands must still parse with the current options
and run committed files only."""
import glob
import os
import re
import shlex

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _commands():
    cmds = set()
    for path in glob.glob(os.path.join(ROOT, "profiles", "*.md")):
        text = open(path).read()
        for m in re.finditer(r"python bench\.py([^>&|\n]*)", text):
            cmds.add((os.path.basename(path), m.group(1).strip()))
    return sorted(cmds)


def test_profiles_name_their_commands():
    assert _commands(), "no bench.py commands found under profiles/"


@pytest.mark.parametrize("name,args", _commands())
def test_profile_command_parses(name, args):
    import bench
    bench.build_parser().parse_args(shlex.split(args))


def test_profiles_run_committed_files_only():
    for path in glob.glob(os.path.join(ROOT, "profiles", "*.md")):
        text = open(path).read()
        assert "_work/" not in text, path
        assert "/root/" not in text, path
