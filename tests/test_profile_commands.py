"""The commands the profile summaries under profiles/ give still parse with bench.py's options, so that every
committed measurement can be reproduced as written."""
import glob
import importlib.util
import os
import re
import shlex
import sys

import pytest

import helpers as H

PROFILES = sorted(glob.glob(os.path.join(H.ROOT, "profiles", "*.md")))


def _bench():
    spec = importlib.util.spec_from_file_location("bench_cli", os.path.join(H.ROOT, "bench.py"))
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


def _commands(path):
    text = open(path).read().replace("\\\n", " ")
    return sorted({m.strip() for m in re.findall(r"python bench\.py([^`\n&|>]*)", text)})


@pytest.mark.parametrize("path", PROFILES, ids=[os.path.basename(p) for p in PROFILES])
def test_profile_commands_parse(path, monkeypatch):
    cmds = _commands(path)
    assert cmds, f"{path} gives no bench.py command"
    bench = _bench()
    for c in cmds:
        monkeypatch.setattr(sys, "argv", ["bench.py"] + shlex.split(c))
        bench.parse_args()              # exits (SystemExit) on an unknown option
