"""Parameter handling mirrors src/par.c (defaults, -par files, --k=v, --k v,
bare --flag, -unpol / -quench / -check, unknown keys ignored, the
max_pol_frac quirk of src/model_radiation.c:94-95, histogram refusal)."""
import pytest

import ipole_b200 as ip


def test_defaults_match_reference():
    p = ip.Params()
    assert (p.rcam, p.thetacam, p.nx, p.ny, p.eps, p.maxnstep, p.emission_type) == (1000., 90., 160, 160, 0.01, 50000, 4)
    assert (p.refine_rel, p.refine_abs, p.refine_cut, p.nx_min, p.target_nturns) == (0.1, 1e-5, 0.0, -1, -1)
    assert p.dsource == 16.9e6 and p.MBH_solar == 6.2e9 and p.trat_large == 40. and p.sigma_cut == 1.
    assert p.dump == "dump.h5" and p.rmax_geo == 100. and p.rmin_geo == 1.


def test_command_line_forms(tmp_path):
    par = tmp_path / "a.par"
    par.write_text("# comment\nnx 64\nfreqcgs 230.e9\nthetacam 17\nunknown_key 3\n")
    p = ip.Params.from_args(["-par", str(par), "--nx=32", "--ny", "48", "--qu_conv", "--M_unit=3e26", "-unpol"])
    assert p.nx == 32 and p.ny == 48 and p.freqcgs == 230e9 and p.thetacam == 17
    assert p.qu_conv == 1 and p.only_unpolarized == 1 and p.M_unit == 3e26
    # as in src/par.c:194-203, a bare --flag takes the next argument as its value unless that starts with "--"
    assert ip.Params.from_args(["--qu_conv", "-unpol"]).qu_conv == 0


def test_order_dependent_overwrite(tmp_path):
    par = tmp_path / "b.par"
    par.write_text("nx 10\n")
    assert ip.Params.from_args(["--nx=5", "-par", str(par)]).nx == 10
    assert ip.Params.from_args(["-par", str(par), "--nx=5"]).nx == 5


def test_fov_sets_both_axes_and_flags():
    p = ip.Params.from_args(["--fov=120", "-quench", "-check"])
    assert p.fovx_dsource == 120 and p.fovy_dsource == 120 and p.quench_output == 1 and p.perform_check == 1


def test_max_pol_frac_quirk():
    p = ip.Params.from_args(["--max_pol_frac_e=0.5"])
    assert p.powerlaw_p == 0.5


def test_mdot_sets_unit_mass():
    assert ip.Params.from_args(["--mdot=1e-7"]).M_unit == 1.0


def test_histogram_request_is_refused():
    with pytest.raises(ip.IpgError) as e:
        ip.Params.from_args(["--histo=1"])
    assert e.value.code == ip.IPG_E_ARG


def test_missing_par_file():
    with pytest.raises(ip.IpgError) as e:
        ip.Params.from_args(["-par", "/nonexistent/file.par"])
    assert e.value.code == ip.IPG_E_IO


def test_mixed_precision_keys(tmp_path):
    """mixed_records and fp32_step (keys of this implementation, no reference
    counterpart) are off by default and read from the command line and from
    -par files like any other integer key."""
    p = ip.Params()
    assert p.mixed_records == 0 and p.fp32_step == 0
    par = tmp_path / "m.par"
    par.write_text("fp32_step 1\n")
    q = ip.Params.from_args(["--mixed_records=1", "-par", str(par)])
    assert q.mixed_records == 1 and q.fp32_step == 1
