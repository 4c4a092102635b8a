"""The oracle port against the reference's known-answer outputs (CPU only).

Every case restates a system test of the reference; its expected stdout is
the reference's own test_<name>.manual.ref.c output, committed under
tests/golden/. The port must reproduce it byte for byte.
"""
import pytest

from tests.golden import cases as C

CASES = C.case_list()


@pytest.mark.parametrize("name", sorted(CASES))
def test_port_matches_golden(name):
    case = CASES[name]
    out = C.run_oracle(case)
    assert C.dump_text(out, case["fmt"]) == C.golden_text(name)


def test_golden_manifest_digests():
    import hashlib
    import json
    import os
    with open(os.path.join(C.HERE, "manifest.json")) as f:
        man = json.load(f)
    from tests.golden import dsl_cases
    assert set(man) == set(CASES) | set(dsl_cases.extra_cases()) | set(dsl_cases.user_cases())
    for name, rec in man.items():
        assert hashlib.sha256(C.golden_text(name).encode()).hexdigest() == rec["sha256"]
