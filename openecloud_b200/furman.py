"""Furman-Pivi secondary-emission parameters (no GPU framework needed).

The copper and stainless-steel tables of copperMod / stainlessMod
(particleEmitter.pyx:107-152) and the oec_furman_t structure the emission
kernel reads (include/oec.h).
"""
import ctypes

from .constants import pi

_D = ctypes.c_double


class Furman_t(ctypes.Structure):
    _fields_ = [(n, _D) for n in ("p1EInf", "p1Ehat", "eEHat", "w", "p", "e1", "e2", "p1RInf", "eR", "r", "r1",
                                  "r2", "q", "sigmaE", "deltaTSHat", "s", "eHat0", "t1", "t2", "t3", "t4",
                                  "theta0max", "deltaERmax")] + \
               [("epsN", _D * 10), ("pSmallN", _D * 10), ("particle_mass", _D), ("m", ctypes.c_int32),
                ("scaleSigmaE", ctypes.c_int32), ("compat_last", ctypes.c_int32), ("reserved", ctypes.c_int32)]


# Parameter tables of particleEmitter.pyx:107-128 (stainless) and :130-152 (copper).
STAINLESS = dict(p1EInf=0.07, p1Ehat=0.5, eEHat=0., w=100., p=0.9, e1=0.26, e2=2., q=0.4, sigmaE=1.9,
                 p1RInf=0.74, eR=40., r=1., r1=0.26, r2=2., deltaTSHat=1.22, s=1.813, eHat0=310., t3=0.7,
                 t4=1., t1=0.66, t2=0.8,
                 epsN=[3.9, 6.2, 13., 8.8, 6.25, 2.25, 9.2, 5.3, 17.8, 10.],
                 pSmallN=[1.6, 2., 1.8, 4.7, 1.8, 2.4, 1.8, 1.8, 2.3, 1.8])
COPPER = dict(p1EInf=0.02, p1Ehat=0.496, eEHat=0., w=60.86, p=1., e1=0.26, e2=2., sigmaE=2., p1RInf=0.2,
              eR=0.041, r=0.104, q=0.5, r1=0.26, r2=2., deltaTSHat=1.8848, s=1.54, eHat0=276.8, t3=0.7, t4=1.,
              t1=0.66, t2=0.8,
              epsN=[2.5, 3.3, 2.5, 2.5, 2.8, 1.3, 1.5, 1.5, 1.5, 1.5],
              pSmallN=[1.5, 1.75, 1., 3.75, 8.5, 11.5, 2.5, 3., 2.5, 3.])


def furman_params(material="copper", seyMax=-1., reflec=-1.):
    """Model parameters as copperMod / stainlessMod set them."""
    if material == "stainless":
        t = dict(STAINLESS)
    elif material == "copper":
        t = dict(COPPER)
    else:
        raise ValueError('Material "' + str(material) + '" not implemented.')
    t["theta0max"] = 84. * pi / 180
    t["deltaERmax"] = 0.99
    if seyMax >= 0.5:
        t["deltaTSHat"] = seyMax - t["p1RInf"] - t["p1EInf"]
    if reflec >= 0.:
        t["p1Ehat"] = reflec
    return t


def furman_struct(params, particle_mass, m=10, scaleSigmaE=0, compat=True):
    """The oec_furman_t of a parameter table (furman_params)."""
    f = Furman_t()
    for k, v in params.items():
        if k in ("epsN", "pSmallN"):
            getattr(f, k)[:] = [float(x) for x in v]
        else:
            setattr(f, k, float(v))
    f.particle_mass = float(particle_mass)
    f.m = int(m)
    f.scaleSigmaE = int(scaleSigmaE)
    f.compat_last = 1 if compat else 0
    return f
