"""Reader of the reference's run-parameter file `sharpclaw.data`, in the
order src/main.f90:61-122 reads it, so a run set up for the reference (by its
setrun.py) can be started here from the same file.

The file is what setrun.py writes: a comment header, then one record per
item, `value(s) =: name (description)`.  As the Fortran list-directed reads
do, each read starts at the next non-blank record and takes as many values
as it asks for, continuing onto the following records when one record holds
fewer (the rest of its last record is skipped); blank records and `#` lines
are skipped.  The plugin id and its physical constants
(the app's setprob.data) are not in this file: pass them to `claw_params`.
"""
from __future__ import annotations


def _records(text: str):
    for line in text.splitlines():
        body = line.split("=:", 1)[0].strip()
        if not body or line.lstrip().startswith("#"):
            continue
        yield body.replace(",", " ").replace("d", "e").replace("D", "E").split()


def read_sharpclaw_data(path: str) -> dict:
    """The parameters of sharpclaw.data as a dict (names as main.f90 uses
    them; `nx`, `xlower`, `xupper` per dimension, `mthbc` per side)."""
    with open(path) as f:
        recs = _records(f.read())

    def nvals(n, conv=float):
        # one list-directed read of n values (main.f90:78 tout(1:nout),
        # :106 mthlim(1:mwaves)): records are consumed until n values are read
        vals = []
        while len(vals) < n:
            try:
                vals += next(recs)
            except StopIteration:
                raise ValueError(f"{path}: end of file after {len(vals)} of {n} values") from None
        return [conv(v) for v in vals[:n]]

    def nxt(n=1, conv=float):
        out = nvals(n, conv)
        return out if n > 1 else out[0]

    def ival(v):
        return int(float(v))

    d = {}
    d["ndim"] = nxt(conv=ival)                                          # :61
    d["nx"] = [nxt(conv=ival) for _ in range(d["ndim"])]                # :63-65
    d["nout"] = nxt(conv=ival)                                          # :70
    d["outstyle"] = nxt(conv=ival)                                      # :71
    if d["outstyle"] == 1:                                              # :72-84
        d["tfinal"] = nxt()
    elif d["outstyle"] == 2:
        d["tout"] = nvals(d["nout"])
    elif d["outstyle"] == 3:
        d["nstepout"], d["nstop"] = nxt(2, ival)
        d["nout"] = d["nstop"]
    else:
        raise ValueError(f"{path}: outstyle must be 1, 2 or 3")
    for k in ("dt_initial", "dt_max", "cfl_max", "cfl_desired"):        # :86-89
        d[k] = nxt()
    d["max_steps"] = nxt(conv=ival)                                     # :90
    for k in ("dt_variable", "time_integrator", "verbosity", "src_term", "mcapa", "maux",
              "tfluct_solver", "char_decomp", "meqn", "mwaves", "lim_type"):   # :93-104
        d[k] = nxt(conv=ival)
    d["mthlim"] = nvals(d["mwaves"], ival)                              # :106
    d["t0"] = nxt()                                                     # :109
    d["xlower"], d["xupper"] = [], []
    for _ in range(d["ndim"]):                                          # :112-115
        d["xlower"].append(nxt())
        d["xupper"].append(nxt())
    d["mbc"] = nxt(conv=ival)                                           # :118
    d["mthbc"] = [nxt(conv=ival) for _ in range(2 * d["ndim"])]         # :120-122
    return d


def claw_params(data: dict, rp: int, **plugin) -> "ClawParams":
    """ClawParams of a run described by read_sharpclaw_data, for plugin `rp`
    with its constants (u, gamma, grav, efix, rho, bulk) as keywords.  The
    reference's src_term flag selects nothing (it links the app's src1.f90);
    pass src_term= with an SCL_SRC_* hook instead."""
    from . import ClawParams
    nd = data["ndim"]
    dx = (data["xupper"][0] - data["xlower"][0]) / data["nx"][0]
    kw = dict(rp=rp, mx=data["nx"][0], dx=dx, xlower=data["xlower"][0], ndim=nd, meqn=data["meqn"],
              mwaves=data["mwaves"], maux=data["maux"], mbc=data["mbc"], mcapa=data["mcapa"],
              lim_type=data["lim_type"], char_decomp=data["char_decomp"], tfluct_solver=data["tfluct_solver"],
              mthbc=tuple(data["mthbc"]) + (2,) * (4 - 2 * nd), time_integrator=data["time_integrator"],
              mthlim=tuple(data["mthlim"][:4]) + (1,) * max(0, 4 - len(data["mthlim"])))
    if nd == 2:
        kw.update(my=data["nx"][1], dy=(data["xupper"][1] - data["xlower"][1]) / data["nx"][1],
                  ylower=data["xlower"][1])
    kw.update(plugin)
    return ClawParams(**kw)


def run_settings(data: dict) -> dict:
    """Keyword arguments of Solver.run_frames for the run's output loop."""
    out = dict(t0=data["t0"], dt_initial=data["dt_initial"], cfl_max=data["cfl_max"],
               cfl_desired=data["cfl_desired"], dt_max=data["dt_max"], max_steps=data["max_steps"],
               dt_variable=data["dt_variable"])
    if data["outstyle"] == 1:
        out.update(nout=data["nout"], tfinal=data["tfinal"])
    elif data["outstyle"] == 2:
        out.update(tout=data["tout"])
    else:
        raise ValueError("outstyle 3 (single steps) has no output-loop equivalent here; use Solver.rk_step")
    return out
