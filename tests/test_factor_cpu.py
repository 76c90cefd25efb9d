"""Block factorizations and truncation (src/factorizations/) on host tensors: the selection
logic and the assembly of the factors, checked against numpy and the oracle's restatement of the
truncation rules. The device run is tests/test_gpu_factor.py."""
import pytest

import factor_checks as FC


@pytest.mark.parametrize("cplx", [False, True])
def test_svd(cplx):
    FC.check_svd("cpu", cplx)


def test_truncation():
    FC.check_truncation("cpu")


@pytest.mark.parametrize("cplx", [False, True])
def test_qr_lq(cplx):
    FC.check_qr_lq("cpu", cplx)


@pytest.mark.parametrize("cplx", [False, True])
def test_eigh(cplx):
    FC.check_eigh("cpu", cplx)
