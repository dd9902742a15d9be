"""The committed profile summaries: short text files, each naming the command that made
it. Every ncu command in them leaves the GPU's clocks alone (`--clock-control none`), and
captures either the one-pass launch list or a bounded number of launches of one kernel."""
import glob
import os
import re

from conftest import ROOT

PROFILES = sorted(glob.glob(os.path.join(ROOT, "profiles", "*")))


def test_profiles_are_short_text_summaries():
    assert PROFILES
    for path in PROFILES:
        assert path.endswith((".md", ".txt")), path
        assert os.path.getsize(path) < 16 * 1024, path


def test_every_ncu_command_keeps_the_clocks_and_is_bounded():
    for path in PROFILES:
        text = open(path).read()
        cmds = [line for line in text.splitlines() if re.match(r"\s*ncu\s", line)]
        assert cmds, f"{path}: names no ncu command"
        for cmd in cmds:
            assert "--clock-control none" in cmd, (path, cmd)
            if "-i " in cmd:  # reading a report back, no capture
                continue
            launch_list = "--metrics gpu__time_duration.sum" in cmd and "--set" not in cmd
            if not launch_list:
                assert re.search(r"-k\s", cmd), (path, "a multi-pass capture names one kernel")
                m = re.search(r"-c\s+(\d+)", cmd)
                assert m and int(m.group(1)) <= 4, (path, "a multi-pass capture takes 1-4 launches")
