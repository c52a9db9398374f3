"""config.toml schema and validation (src/lib.rs:34-117)."""
import pytest

from spectral_rs_b200.config import Config, ConfigError

BASE = """
[setup]
t_final = 500

[params]
size_x = 2048
size_y = 256
delta = 64
dt = 0.1
c = 3.0
dens = 2
gamma_inj = 10.0
n_pass = 4

[output]
track_prtls = false
track_interval = 100
write_output = false
output_interval = 50
stride = 1
istep = 1
"""


def _cfg(tmp_path, text):
    p = tmp_path / "config.toml"
    p.write_text(text)
    return Config.new(str(p))


def test_reference_config_parses(tmp_path):
    cfg = _cfg(tmp_path, BASE)
    assert cfg.params.size_x == 2048 and cfg.setup.t_final == 500
    # additive keys default to the reference's behaviour
    assert cfg.params.mass_ratio == 1.0 and cfg.params.vth == 1e-3 and not cfg.params.periodic_x
    sp = cfg.species_list()
    assert [(s.charge, s.mass) for s in sp] == [(1.0, 1.0), (-1.0, 1.0)]


@pytest.mark.parametrize("edit,msg", [
    (("size_x = 2048", "size_x = 2047"), "x direction must be even"),
    (("size_y = 256", "size_y = 255"), "y direction must be even"),
    (("delta = 64", "delta = 1024"), "Delta must be less"),
    (("gamma_inj = 10.0", "gamma_inj = 1.0"), "Lorentz factor"),
    (("istep = 1", "istep = 3"), "divisible"),
])
def test_validation_errors(tmp_path, edit, msg):
    with pytest.raises(ConfigError, match=msg):
        _cfg(tmp_path, BASE.replace(*edit))


def test_missing_key_is_an_error(tmp_path):
    with pytest.raises(ConfigError):
        _cfg(tmp_path, BASE.replace("n_pass = 4\n", ""))


def test_missing_file():
    with pytest.raises(ConfigError, match="Could not open"):
        Config.new("/nonexistent/config.toml")


def test_species_tables(tmp_path):
    text = BASE + """
[[species]]
charge = -1.0
mass = 1.0
vth = 0.01
ppc = 32
drift_gamma = 1.0206
drift_sign = 1.0

[[species]]
charge = -1.0
mass = 1.0
vth = 0.01
ppc = 32
drift_gamma = 1.0206
drift_sign = -1.0
"""
    cfg = _cfg(tmp_path, text)
    assert len(cfg.species_list()) == 2 and cfg.species_list()[1].drift_sign == -1.0
