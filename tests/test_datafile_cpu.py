"""The reader of sharpclaw.data (src/main.f90:61-122): a run set up for the
reference starts here from the same file.  The files below are written in
the format setrun.py produces (header, `value =: name (description)`
records, blank lines between groups)."""
import sharpclaw_b200 as S

HEADER = "#" * 56 + "\n### generated file ###\n" + "#" * 56 + "\n\n"


def _write(path, records):
    lines = [HEADER]
    for rec in records:
        lines.append("" if rec is None else f"{rec[0]:<26}=: {rec[1]}")
    path.write_text("\n".join(lines) + "\n")


def test_read_1d_outstyle1(tmp_path):
    f = tmp_path / "sharpclaw.data"
    _write(f, [("1", "ndim"), ("1500", "mx"), None, ("10", "nout"), ("1", "outstyle"),
               ("2.2000000000000002", "tfinal"), None, ("0.025", "dt_initial"), ("9.99e+98", "dt_max"),
               ("0.4", "cfl_max"), ("0.35", "cfl_desired"), ("50000", "max_steps"), None,
               ("1", "dt_variable"), ("4", "time_integrator"), ("0", "verbosity"), ("0", "src_term"),
               ("0", "mcapa"), ("0", "maux"), ("0", "tfluct_solver"), ("2", "char_decomp"), None,
               ("3", "meqn"), ("3", "mwaves"), ("2", "lim_type"), ("5 5 5", "mthlim"), None,
               ("0.0", "t0"), ("-5.0", "xlower"), ("5.0", "xupper"), None, ("3", "mbc"),
               ("1", "mthbc_xlower"), ("1", "mthbc_xupper"), ("0", "restart")])
    d = S.read_sharpclaw_data(str(f))
    assert d["ndim"] == 1 and d["nx"] == [1500] and d["nout"] == 10 and d["tfinal"] == 2.2000000000000002
    assert d["cfl_max"] == 0.4 and d["max_steps"] == 50000 and d["time_integrator"] == 4
    assert d["mthlim"] == [5, 5, 5] and d["xlower"] == [-5.0] and d["mthbc"] == [1, 1]
    p = S.claw_params(d, S.RP_EULER, gamma=1.4)
    assert p.mx == 1500 and abs(p.dx - 10.0 / 1500) < 1e-15 and p.xlower == -5.0
    assert p.char_decomp == 2 and p.tfluct_solver == 0 and p.time_integrator == 4 and p.efix == 1
    assert tuple(p.mthbc[:2]) == (1, 1) and p.gamma == 1.4
    r = S.run_settings(d)
    assert r == dict(t0=0.0, dt_initial=0.025, cfl_max=0.4, cfl_desired=0.35, dt_max=9.99e98, max_steps=50000,
                     dt_variable=1, nout=10, tfinal=2.2000000000000002)


def test_read_2d_outstyle2(tmp_path):
    f = tmp_path / "sharpclaw.data"
    _write(f, [("2", "ndim"), ("40", "mx"), ("30", "my"), ("3", "nout"), ("2", "outstyle"),
               ("0.1 0.25 0.5", "tout"), ("0.01", "dt_initial"), ("1d99", "dt_max"), ("0.9", "cfl_max"),
               ("0.8", "cfl_desired"), ("500", "max_steps"), ("1", "dt_variable"), ("3", "time_integrator"),
               ("0", "verbosity"), ("0", "src_term"), ("0", "mcapa"), ("0", "maux"), ("1", "tfluct_solver"),
               ("1", "char_decomp"), ("3", "meqn"), ("3", "mwaves"), ("2", "lim_type"), ("4 4 4", "mthlim"),
               ("0.0", "t0"), ("-2.5", "xlower"), ("2.5", "xupper"), ("-1.5", "ylower"), ("1.5", "yupper"),
               ("3", "mbc"), ("3", "mthbc_xlower"), ("1", "mthbc_xupper"), ("2", "mthbc_ylower"),
               ("2", "mthbc_yupper")])
    d = S.read_sharpclaw_data(str(f))
    assert d["nx"] == [40, 30] and d["tout"] == [0.1, 0.25, 0.5] and d["dt_max"] == 1e99
    assert d["xlower"] == [-2.5, -1.5] and d["xupper"] == [2.5, 1.5] and d["mthbc"] == [3, 1, 2, 2]
    p = S.claw_params(d, S.RP_SW2D, grav=1.0)
    assert (p.mx, p.my, p.ndim) == (40, 30, 2) and p.dx == 5.0 / 40 and p.dy == 3.0 / 30
    assert p.ylower == -1.5 and tuple(p.mthbc) == (3, 1, 2, 2) and p.char_decomp == 1
    assert S.run_settings(d)["tout"] == [0.1, 0.25, 0.5]


def test_list_directed_reads_continue_across_records(tmp_path):
    """tout(1:nout) (main.f90:78) and mthlim(1:mwaves) (:106) are list-directed
    reads: when one record holds fewer values they continue onto the next
    records, and every later item is read from the record after them."""
    f = tmp_path / "sharpclaw.data"
    lines = [HEADER, "1 =: ndim", "200 =: mx", "5 =: nout", "2 =: outstyle",
             "0.1 0.2", "0.3", "0.4 0.5 =: tout", "0.01 =: dt_initial", "1e99 =: dt_max", "0.9 =: cfl_max",
             "0.8 =: cfl_desired", "500 =: max_steps", "1 =: dt_variable", "3 =: time_integrator",
             "0 =: verbosity", "0 =: src_term", "0 =: mcapa", "0 =: maux", "0 =: tfluct_solver",
             "2 =: char_decomp", "3 =: meqn", "3 =: mwaves", "2 =: lim_type", "1 2", "3 =: mthlim",
             "0.0 =: t0", "-5.0 =: xlower", "5.0 =: xupper", "3 =: mbc", "1 =: mthbc_xlower",
             "1 =: mthbc_xupper"]
    f.write_text("\n".join(lines) + "\n")
    d = S.read_sharpclaw_data(str(f))
    assert d["tout"] == [0.1, 0.2, 0.3, 0.4, 0.5]
    assert d["dt_initial"] == 0.01 and d["max_steps"] == 500
    assert d["mthlim"] == [1, 2, 3] and d["t0"] == 0.0 and d["xlower"] == [-5.0] and d["mthbc"] == [1, 1]


def test_truncated_file_is_an_error(tmp_path):
    import pytest
    f = tmp_path / "sharpclaw.data"
    f.write_text(HEADER + "1 =: ndim\n200 =: mx\n4 =: nout\n2 =: outstyle\n0.1 0.2 =: tout\n")
    with pytest.raises(ValueError, match="end of file"):
        S.read_sharpclaw_data(str(f))
