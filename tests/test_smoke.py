"""The build's smoke check (one closest-hit query of the Cornell fixture against the reference's
answers) runs as a GPU test too, so that its checker is exercised with every GPU suite."""

import pytest


@pytest.mark.gpu
def test_smoke_entry_point(gpu_lib, capsys):
    import __graft_entry__ as entry

    entry.smoke()
    assert "Cornell rays match the reference closest hits" in capsys.readouterr().out
