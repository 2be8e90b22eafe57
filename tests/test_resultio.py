"""Vm.pt written row by row (torchcor_b200/simulator/resultio.py) must be the file
torch.save writes: torch.load returns the same tensor and every record's CRC-32
checks (zipfile.testzip)."""
import zipfile

import pytest
import torch

from torchcor_b200.simulator.resultio import StreamedTensorFile


@pytest.mark.parametrize("shape", [(7, 1000), (1, 5), (4, 3, 5), (101, 4099)])
def test_rows_in_order_make_the_torch_save_file(tmp_path, shape):
    g = torch.Generator().manual_seed(1)
    x = torch.randn(shape, generator=g)
    p = tmp_path / "Vm.pt"
    f = StreamedTensorFile(p, shape, torch.float32)
    for i in range(shape[0]):
        f.write_row(i, x[i].contiguous().numpy())
    f.close()
    assert torch.equal(torch.load(p), x)
    with zipfile.ZipFile(p) as z:
        assert z.testzip() is None
    # the same records as torch.save's own file of the tensor
    q = tmp_path / "ref.pt"
    torch.save(x, q)
    with zipfile.ZipFile(p) as a, zipfile.ZipFile(q) as b:
        ia = {i.filename.split("/", 1)[1]: i for i in a.infolist()}
        ib = {i.filename.split("/", 1)[1]: i for i in b.infolist()}
        assert ia.keys() == ib.keys()
        for k in ia:
            if k != ".data/serialization_id":          # a fresh id per save
                assert a.read(ia[k]) == b.read(ib[k]), k
                assert ia[k].CRC == ib[k].CRC, k


def test_out_of_order_or_missing_rows_are_errors(tmp_path):
    x = torch.ones(3, 8)
    f = StreamedTensorFile(tmp_path / "a.pt", x.shape)
    with pytest.raises(ValueError):
        f.write_row(1, x[1].numpy())
    f.write_row(0, x[0].numpy())
    with pytest.raises(ValueError):
        f.write_row(1, torch.ones(9).numpy())               # wrong size
    with pytest.raises(RuntimeError):
        f.close()                                            # rows 1 and 2 missing
    g = StreamedTensorFile(tmp_path / "b.pt", x.shape)
    g.write_row(0, x[0].numpy())
    g.abandon()                                              # no CRC: the file does not check
    with zipfile.ZipFile(tmp_path / "b.pt") as z:
        assert z.testzip() is not None
