"""Material models (fenris/src/solid/materials.rs) as POD descriptors.

The kernels evaluate the models; these classes only carry the parameters,
mirroring the reference's `From<YoungPoisson>` / `From<LameParameters>`
constructors.
"""
from dataclasses import dataclass

from . import _capi


@dataclass(frozen=True)
class YoungPoisson:
    young: float
    poisson: float


@dataclass(frozen=True)
class LameParameters:
    mu: float
    lam: float

    @staticmethod
    def from_young_poisson(yp):
        """LameParameters::from(YoungPoisson), materials.rs:27-38 (reference
        conversion, lambda = 0.5 mu nu / (1 - 2 nu))."""
        mu, lam = _capi.C.c_double(), _capi.C.c_double()
        _capi.check(_capi.lib().hoefem_lame_from_young_poisson(yp.young, yp.poisson, _capi.C.byref(mu),
                                                               _capi.C.byref(lam)))
        return LameParameters(mu.value, lam.value)


def _lame(params):
    if isinstance(params, LameParameters):
        return params
    if isinstance(params, YoungPoisson):
        return LameParameters.from_young_poisson(params)
    raise TypeError("expected YoungPoisson or LameParameters")


class _MaterialBase:
    kind = None

    def __init__(self, params):
        self.lame = _lame(params)

    def descriptor(self):
        return _capi.Material(self.kind, self.lame.mu, self.lame.lam)

    def __repr__(self):
        return "%s(mu=%g, lambda=%g)" % (type(self).__name__, self.lame.mu, self.lame.lam)


class StableNeoHookeanMaterial(_MaterialBase):
    """Stable Neo-Hookean (Smith et al. 2018), materials.rs:221-377."""
    kind = _capi.MAT_SNH


class StVKMaterial(_MaterialBase):
    """St. Venant-Kirchhoff, materials.rs:177-219."""
    kind = _capi.MAT_STVK
