"""Where the reference's sources are read from -- test infrastructure and
build recipes only (oracle/Makefile uses the same variable).

$GMK_REFERENCE names the checkout; without it the default checkout location
below is used.  Nothing on the GPU side reads it: the built oracles under
oracle/_ref and the committed fixtures under tests/golden travel instead.
"""
import os

REFERENCE = os.environ.get("GMK_REFERENCE") or "/root/reference"


def ref_path(*parts: str) -> str:
    """A path inside the reference checkout."""
    return os.path.join(REFERENCE, *parts)


def have_reference() -> bool:
    """True when the reference's CPU enumerator sources are present."""
    return os.path.isdir(ref_path("baselines", "MaximalBiPlex"))
