"""Host-side argument checks of the Python engine (CPU): shapes are checked
before any pointer reaches the C ABI, so a short array is never read past its
end on the host or the device."""
import numpy as np
import pytest

from swiftimpute_b200 import _native as N
from swiftimpute_b200.engine import Engine, _job_layout


def test_job_layout_offsets_and_length_check():
    regions = [(0, 10, 8, N.INDEX_GLOBAL), (5, 8, 4, N.INDEX_REGION)]
    jobs = [(1, np.zeros(3, np.uint8), 0), (0, np.zeros(10, np.uint8), 1), (1, np.zeros(3, np.uint8), 2)]
    lens, offs = _job_layout(regions, jobs)
    assert lens == [3, 10, 3] and offs.tolist() == [0, 3, 13, 16]
    with pytest.raises(ValueError, match="job 1"):
        _job_layout(regions, [jobs[0], (0, np.zeros(9, np.uint8), 1)])
    # an unknown region or an empty one has length 0; the C ABI refuses the batch
    assert _job_layout(regions, [(7, np.zeros(0, np.uint8), 0)])[0] == [0]
    assert _job_layout([(5, 3, 8, N.INDEX_GLOBAL)], [(0, np.zeros(0, np.uint8), 0)])[0] == [0]
    with pytest.raises(ValueError):
        _job_layout(regions, [(7, np.zeros(4, np.uint8), 0)])


def test_impute_checks_the_code_matrix_shape():
    e = Engine.__new__(Engine)  # no device context: the check comes first
    e.h, e.lib, e.M, e.N = None, None, 12, 40
    with pytest.raises(ValueError, match="shape"):
        e.impute(np.zeros((3, 11), np.uint8))
    with pytest.raises(ValueError, match="shape"):
        e.impute(np.zeros((3, 12), np.float32), gl=True)
    with pytest.raises(ValueError, match="shape"):
        e.impute(np.zeros(12, np.uint8))
