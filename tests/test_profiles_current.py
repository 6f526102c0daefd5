"""Every profile summary under profiles/ names the engine build it was
captured on, and that build is the one the repository's stage-kernel sources
make (pangu_b200.build.source_hash()): the committed figures describe the
committed kernels. bench.py refuses a stale summary at run time; this test
catches one before it is committed."""
import os
import re

from pangu_b200 import build

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PROFILES = os.path.join(ROOT, "profiles")


def _builds(path):
    text = open(path).read()
    found = re.findall(r"^build ([0-9a-f]{16})$", text, re.M)
    found += re.findall(r"engine (?:kernel )?sources ([0-9a-f]{16})", text)
    return set(found)


def test_every_profile_names_the_current_build():
    want = build.source_hash()
    names = sorted(os.listdir(PROFILES))
    assert names, "no profile summaries"
    for name in names:
        got = _builds(os.path.join(PROFILES, name))
        assert got, f"{name} names no build"
        assert got == {want}, (name, got, want)


def test_profiles_are_text_summaries():
    for name in os.listdir(PROFILES):
        assert name.endswith((".md", ".txt")), name
        assert os.path.getsize(os.path.join(PROFILES, name)) < 64 * 1024, name
