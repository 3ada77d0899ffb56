"""CPU check: the header-only C++ index-label front end compiles and links
against the C ABI (no GPU needed)."""
import subprocess

import pytest

from frontend_build import build


def test_frontend_header_compiles_and_links():
    try:
        out = build()
    except subprocess.CalledProcessError as e:
        pytest.fail(f"front end failed to build:\n{e.stderr}")
    assert out.exists()
