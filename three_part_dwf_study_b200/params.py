"""parameters.txt reader with the reference's semantics (common/config.hpp:11-109).

``key = value`` lines; ``#`` starts a comment; blank lines are skipped. A line
without ``=`` or with an empty key or value is an error naming file:line
(config.hpp:32-46). A missing key raises "Missing required parameter: <key>"
(:90-96); a numeric value with trailing characters raises "Invalid numeric
value for <key>: <value>" (:99-106). Later duplicates overwrite earlier ones.
"""
import re
from pathlib import Path

_INT = re.compile(r"^\s*[+-]?\d+")
_UINT = re.compile(r"^\s*[+-]?\d+")
_REAL = re.compile(r"^\s*[+-]?(?:(?:\d+\.?\d*|\.\d+)(?:[eE][+-]?\d+)?|inf(?:inity)?|nan)",
                   re.IGNORECASE)


class ConfigError(RuntimeError):
    pass


class TextConfig:
    def __init__(self, filename="parameters.txt", text=None):
        self.filename = str(filename)
        if text is None:
            try:
                text = Path(filename).read_text()
            except OSError:
                raise ConfigError(f"Cannot open parameter file: {filename}")
        self.values = {}
        for n, raw in enumerate(text.splitlines(), 1):
            line = raw.split("#", 1)[0].strip()
            if not line:
                continue
            if "=" not in line:
                raise ConfigError(f"{self.filename}:{n}: expected key = value")
            key, value = line.split("=", 1)
            key, value = key.strip(), value.strip()
            if not key or not value:
                raise ConfigError(f"{self.filename}:{n}: empty key or value")
            self.values[key] = value

    def _require(self, key):
        if key not in self.values:
            raise ConfigError(f"Missing required parameter: {key}")
        return self.values[key]

    def _parse(self, key, rx, conv):
        value = self._require(key)
        m = rx.match(value)
        if not m:
            raise ConfigError(f"Invalid numeric value for {key}: {value}")
        if m.end() != len(value):
            raise ConfigError(f"Invalid numeric value for {key}: {value}")
        return conv(m.group(0))

    def integer(self, key):
        return self._parse(key, _INT, int)

    def unsigned_integer(self, key):
        v = self._parse(key, _UINT, int)
        # std::stoull wraps a leading minus sign modulo 2^64
        return v % (1 << 64)

    def real(self, key):
        return self._parse(key, _REAL, float)

    def text(self, key):
        return self._require(key)

    def get(self, key, default, kind="real"):
        """Additive keys (absent from the reference) fall back to a default
        that reproduces the reference's behaviour."""
        if key not in self.values:
            return default
        return getattr(self, kind)(key)


def dwf_parameters(cfg):
    """The domain-wall parameter table (domain_wall/include/parameters.hpp:7-41)."""
    p = {
        "Nt": cfg.integer("dwf.Nt"), "Nx": cfg.integer("dwf.Nx"), "N5": cfg.integer("dwf.N5"),
        "beta": cfg.real("dwf.beta"), "M5": cfg.real("dwf.M5"), "mf": cfg.real("dwf.mf"),
        "epsilon": cfg.real("dwf.epsilon"), "leapfrog_steps": cfg.integer("dwf.leapfrog_steps"),
        "trajectories": cfg.integer("dwf.trajectories"),
        "thermalization_cut": cfg.integer("dwf.thermalization_cut"),
        "thin": cfg.integer("dwf.thin"),
        "pseudofermion_rtol": cfg.real("dwf.pseudofermion_rtol"),
        "pseudofermion_maxiter": cfg.integer("dwf.pseudofermion_maxiter"),
        "propagator_rtol": cfg.real("dwf.propagator_rtol"),
        "propagator_maxiter": cfg.integer("dwf.propagator_maxiter"),
        "analysis_threads": cfg.integer("analysis.threads"),
        "eta_noise_vectors": cfg.integer("eta.noise_vectors"),
        "eta_flavors": cfg.integer("eta.flavors"),
        "eta_random_seed": cfg.unsigned_integer("eta.random_seed"),
        "max_momentum": cfg.integer("analysis.max_momentum"),
        "random_seed": cfg.unsigned_integer("dwf.random_seed"),
    }
    p["Ndof"] = p["N5"] * p["Nt"] * p["Nx"] * 2
    p["Ngauge"] = 2 * p["Nt"] * p["Nx"]
    return p


def wilson_parameters(cfg):
    """The Wilson parameter table (wilson/include/parameters.hpp:6-44)."""
    p = {
        "Nt": cfg.integer("wilson.Nt"), "Nx": cfg.integer("wilson.Nx"),
        "beta": cfg.real("wilson.beta"), "m0": cfg.real("wilson.m0"),
        "trajectories": cfg.integer("wilson.trajectories"),
        "thermalization_cut": cfg.integer("wilson.thermalization_cut"),
        "thin": cfg.integer("wilson.thin"), "hmc_steps": cfg.integer("wilson.hmc_steps"),
        "trajectory_length": cfg.real("wilson.trajectory_length"),
        "source_t": cfg.integer("wilson.source_t"), "source_x": cfg.integer("wilson.source_x"),
        "time_boundary_sign": cfg.real("wilson.time_boundary_sign"),
        "space_boundary_sign": cfg.real("wilson.space_boundary_sign"),
        "force_cg_tolerance": cfg.real("wilson.force_cg_tolerance"),
        "force_cg_max_iterations": cfg.integer("wilson.force_cg_max_iterations"),
        "measurement_cg_tolerance": cfg.real("wilson.measurement_cg_tolerance"),
        "measurement_cg_max_iterations": cfg.integer("wilson.measurement_cg_max_iterations"),
        "random_seed": cfg.unsigned_integer("wilson.random_seed"),
    }
    p["Ntot"] = p["Nt"] * p["Nx"] * 2
    p["hmc_epsilon"] = p["trajectory_length"] / p["hmc_steps"]
    return p
