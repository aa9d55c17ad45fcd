"""The serving engine's configuration checks that need no GPU: an unknown admission policy is refused."""
from __future__ import annotations

import pytest


def test_unknown_policy_refused():
    pytest.importorskip("torch")
    from woof_nam_b200.serve import RadServer
    with pytest.raises(ValueError, match="policy"):
        RadServer({}, 1368.22, policy="lifo")
