"""The oracle's particle contacts against the reference's contact
known-answer tests (CPU); the same runners check the CUDA path in
test_contacts_gpu.py."""

import pytest

import contact_kats as CK


@pytest.fixture(scope="module")
def cpu(oracle):
    return oracle.OracleBackend(precision=32)


@pytest.mark.parametrize("name", list(CK.ALL))
def test_contact_kat(cpu, name):
    CK.ALL[name](cpu)
