"""Configuration dataclasses with the reference's names and fields
(fv3core/_config.py:129-214): the objects the acoustic-substep classes take."""
import dataclasses


@dataclasses.dataclass(frozen=True)
class RiemannConfig:
    p_fac: float
    a_imp: float
    use_logp: bool
    beta: float


@dataclasses.dataclass(frozen=True)
class DGridShallowWaterLagrangianDynamicsConfig:
    dddmp: float
    d2_bg: float
    d2_bg_k1: float
    d2_bg_k2: float
    d4_bg: float
    ke_bg: float
    nord: int
    n_sponge: int
    grid_type: int
    d_ext: float
    hord_dp: int
    hord_tm: int
    hord_mt: int
    hord_vt: int
    do_f3d: bool
    do_skeb: bool
    d_con: float
    vtdm4: float
    inline_q: bool
    convert_ke: bool
    do_vort_damp: bool
    hydrostatic: bool


@dataclasses.dataclass(frozen=True)
class AcousticDynamicsConfig:
    tau: float
    k_split: int
    n_split: int
    m_split: int
    delt_max: float
    rf_cutoff: float
    rf_fast: bool
    breed_vortex_inline: bool
    use_old_omega: bool
    riemann: RiemannConfig
    d_grid_shallow_water: DGridShallowWaterLagrangianDynamicsConfig

    @property
    def nord(self) -> int:
        return self.d_grid_shallow_water.nord

    @property
    def grid_type(self) -> int:
        return self.d_grid_shallow_water.grid_type

    @property
    def hydrostatic(self) -> bool:
        return self.d_grid_shallow_water.hydrostatic

    @property
    def hord_tm(self) -> int:
        return self.d_grid_shallow_water.hord_tm

    @property
    def p_fac(self) -> float:
        return self.riemann.p_fac

    @property
    def d_ext(self) -> float:
        return self.d_grid_shallow_water.d_ext

    @property
    def d_con(self) -> float:
        return self.d_grid_shallow_water.d_con

    @property
    def beta(self) -> float:
        return self.riemann.beta

    @property
    def use_logp(self) -> bool:
        return self.riemann.use_logp


def baroclinic_dsw_config():
    """D-grid namelist of the baroclinic-wave benchmark configuration
    (fv_core_nml of the reference's examples/wrapped/config/baroclinic.yml)."""
    return DGridShallowWaterLagrangianDynamicsConfig(
        dddmp=0.5, d2_bg=0.0, d2_bg_k1=0.2, d2_bg_k2=0.1, d4_bg=0.15, ke_bg=0.0, nord=3, n_sponge=48,
        grid_type=0, d_ext=0.0, hord_dp=6, hord_tm=6, hord_mt=6, hord_vt=6, do_f3d=False, do_skeb=False,
        d_con=1.0, vtdm4=0.06, inline_q=False, convert_ke=False, do_vort_damp=True, hydrostatic=False,
    )


def baroclinic_acoustic_config(n_split=6, k_split=1):
    return AcousticDynamicsConfig(
        tau=10.0, k_split=k_split, n_split=n_split, m_split=0, delt_max=0.002, rf_cutoff=3000.0, rf_fast=True,
        breed_vortex_inline=False, use_old_omega=True,
        riemann=RiemannConfig(p_fac=0.05, a_imp=1.0, use_logp=False, beta=0.0),
        d_grid_shallow_water=baroclinic_dsw_config(),
    )


@dataclasses.dataclass(frozen=True)
class SatAdjustConfig:
    """The fast saturation adjustment's namelist (fv3core/_config.py:85-110);
    carried by RemappingConfig.  The adjustment itself is not run here:
    LagrangianToEulerian rejects do_sat_adj."""

    hydrostatic: bool
    rad_snow: bool
    rad_rain: bool
    rad_graupel: bool
    tintqs: bool
    sat_adj0: float
    ql_gen: float
    qs_mlt: float
    ql0_max: float
    t_sub: float
    qi_gen: float
    qi_lim: float
    qi0_max: float
    dw_ocean: float
    dw_land: float
    icloud_f: int
    cld_min: float
    tau_i2s: float
    tau_v2l: float
    tau_r2g: float
    tau_l2r: float
    tau_l2v: float
    tau_imlt: float
    tau_smlt: float


@dataclasses.dataclass(frozen=True)
class RemappingConfig:
    """fv3core/_config.py:113-125."""

    fill: bool
    kord_tm: int
    kord_tr: int
    kord_wz: int
    kord_mt: int
    do_sat_adj: bool
    sat_adjust: SatAdjustConfig

    @property
    def hydrostatic(self) -> bool:
        return self.sat_adjust.hydrostatic
