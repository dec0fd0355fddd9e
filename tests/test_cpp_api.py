"""The C++ mirror of the reference's grid/state/step API
(include/deepgreen.hpp) compiles warning-free against the library and keeps
the reference's argument checks, with errors as exceptions (no GPU work)."""
import subprocess

import cpp_api


def test_cpp_mirror_builds_and_validates(tmp_path):
    exe = cpp_api.build(tmp_path)
    r = subprocess.run([str(exe), "validate"], capture_output=True, text=True, timeout=60)
    assert r.returncode == 0, r.stderr
    assert "validate ok" in r.stdout
