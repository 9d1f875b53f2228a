"""Equation descriptors of the hot path, mirroring the reference's
``src/sweep/equations/acoustic.py:48-133`` (``Acoustic``),
``acoustic3d.py:50-185`` (``Acoustic3D``), ``elastic.py:19-310``
(``Elastic``) and ``elastic3d.py:235-332`` (``Elastic3D``): the constructor
keywords, model names and default source / receiver fields the propagator
reads."""
from __future__ import annotations


class _Equation:
    C_NAME = ""
    MODEL_NAMES: tuple = ()
    NDIM = 2
    SOURCE_FIELDS: tuple = ()
    RECEIVER_FIELDS: tuple = ()
    default_pml_type = "cpmlr"

    def __init__(self, spatial_order=4, device="cpu", backend="torch", dim=None):
        if spatial_order % 2 or spatial_order < 2:
            raise ValueError(f"spatial_order must be an even integer >= 2, got {spatial_order}")
        if backend != "torch":
            raise ValueError("sweep_b200 equations run on the torch backend only")
        self.so = int(spatial_order)
        self.spatial_order = self.so
        self.M = self.so // 2
        self.device = device
        self.backend = backend
        self.ndim = self.NDIM

    @property
    def model_names(self):
        return list(self.MODEL_NAMES)

    @property
    def default_source_fields(self):
        return list(self.SOURCE_FIELDS)

    @property
    def default_receiver_fields(self):
        return list(self.RECEIVER_FIELDS)


class Acoustic(_Equation):
    """Second-order 2-D constant-density acoustic wave equation with CPML
    (``u_tt = vp^2 Lap u``; one pressure-like field ``h1``)."""
    C_NAME = "acoustic2d"
    MODEL_NAMES = ("vp",)
    NDIM = 2
    SOURCE_FIELDS = ("h1",)
    RECEIVER_FIELDS = ("h1",)


class Acoustic3D(_Equation):
    """Second-order 3-D constant-density acoustic wave equation with CPML."""
    C_NAME = "acoustic3d"
    MODEL_NAMES = ("vp",)
    NDIM = 3
    SOURCE_FIELDS = ("h1",)
    RECEIVER_FIELDS = ("h1",)


class Elastic(_Equation):
    """First-order 2-D isotropic elastic velocity-stress equation on a
    staggered grid (Virieux 1986): fields vx, vz, sxx, szz, sxz; models
    vp, vs, rho; explosive source (sxx, szz) and (vx, vz) receivers by default."""
    C_NAME = "elastic2d"
    MODEL_NAMES = ("vp", "vs", "rho")
    NDIM = 2
    SOURCE_FIELDS = ("sxx", "szz")
    RECEIVER_FIELDS = ("vx", "vz")
    FIELDS = ("vx", "vz", "sxx", "szz", "sxz")
    default_pml_type = "cpmls"


class Elastic3D(Elastic):
    """First-order 3-D isotropic elastic velocity-stress equation on a
    staggered grid: fields vx, vy, vz, sxx, syy, szz, sxy, sxz, syz; models
    vp, vs, rho; explosive source (sxx, syy, szz) and (vx, vy, vz) receivers
    by default (reference ``equations/elastic3d.py:235-332``)."""
    C_NAME = "elastic3d"
    NDIM = 3
    SOURCE_FIELDS = ("sxx", "syy", "szz")
    RECEIVER_FIELDS = ("vx", "vy", "vz")
    FIELDS = ("vx", "vy", "vz", "sxx", "syy", "szz", "sxy", "sxz", "syz")


class AcousticVTI1st(Elastic):
    """First-order 2-D acoustic VTI velocity-stress equation (Duveneck et al.
    2008) on a staggered grid: fields vx, vz, sH, sV; models vp (vertical),
    Thomsen epsilon and delta, rho (c33 = rho vp^2, c11 = c33 (1 + 2 epsilon),
    c13 = c33 sqrt(1 + 2 delta)); sources on (sH, sV) and vz receivers by
    default (reference ``equations/acoustic_vti_1st.py:244-330``).  No free
    surface, as in the reference."""
    C_NAME = "vti2d"
    MODEL_NAMES = ("vp", "epsilon", "delta", "rho")
    NDIM = 2
    SOURCE_FIELDS = ("sH", "sV")
    RECEIVER_FIELDS = ("vz",)
    FIELDS = ("vx", "vz", "sH", "sV")


class AcousticVTI1st3D(AcousticVTI1st):
    """First-order 3-D acoustic VTI velocity-stress equation (Duveneck et al.
    2008) on a staggered grid: fields vx, vy, vz, sH (= s11 = s22) and sV
    (= s33); the 2-D equation's models and stiffness; sources on (sH, sV) and
    vz receivers by default (reference ``equations/acoustic_vti_1st.py:
    445-600``).  No free surface, as in the reference."""
    C_NAME = "vti3d"
    NDIM = 3
    FIELDS = ("vx", "vy", "vz", "sH", "sV")
