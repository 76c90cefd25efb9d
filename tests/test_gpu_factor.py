"""Block factorizations and truncation (src/factorizations/) on device tensors, checked against
numpy per block and the oracle's restatement of the truncation rules (1e-12 relative)."""
import pytest

import factor_checks as FC

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("cplx", [False, True])
def test_svd(cplx):
    FC.check_svd("cuda", cplx)


def test_truncation():
    FC.check_truncation("cuda")


@pytest.mark.parametrize("cplx", [False, True])
def test_qr_lq(cplx):
    FC.check_qr_lq("cuda", cplx)


@pytest.mark.parametrize("cplx", [False, True])
def test_eigh(cplx):
    FC.check_eigh("cuda", cplx)
