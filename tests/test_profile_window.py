"""The profile-window entry point (`python -m teapotfluidsimulation_b200.profile_window`) imports and
parses its options without a GPU; its preconditioner names map to the C ABI's constants."""
import pytest

from teapotfluidsimulation_b200 import abi, profile_window


def test_help_exits_cleanly(capsys):
    with pytest.raises(SystemExit) as e:
        profile_window.main(["--help"])
    assert e.value.code == 0
    out = capsys.readouterr().out
    for opt in ("--mm", "--start", "--substeps", "--precond"):
        assert opt in out


def test_preconditioner_names():
    assert profile_window.PRECONDS == {
        "cheb": (abi.PRECOND_CHEB, abi.SOLVE_MIXED),
        "mg": (abi.PRECOND_MG, abi.SOLVE_MIXED),
        "box_mg": (abi.PRECOND_BOX_MG, abi.SOLVE_MIXED),
        "mic0": (abi.PRECOND_MIC0, abi.SOLVE_F64),
    }


def test_unknown_preconditioner_is_rejected():
    with pytest.raises(SystemExit) as e:
        profile_window.main(["--precond", "jacobi"])
    assert e.value.code == 2
