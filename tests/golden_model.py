"""Builds oracle models from reference dumps (golden fixtures)."""
import numpy as np

from oracle_lib import Model


def params(g):
    p, ip = g["params"], g["iparams"]
    return dict(dx=p[0], delta=p[1], damping=p[2], rw=p[3], center=p[4:7], total_time=p[7],
                cci=int(ip[0]), cci_mdf=int(ip[1]), mls=int(ip[2]), fgi=int(ip[3]), bdry=int(ip[4]),
                dims=[int(v) for v in ip[5:8]], intg_point=int(ip[8]), total_step=int(ip[9]))


def model_from_golden(g, **over):
    P = params(g)
    n = int(g["n"][0])
    npt = int(g["num_gauss"][0]) if not P["cci"] else 1
    kw = dict(n=n, x=g["coords"], dx=P["dx"], delta=P["delta"], cci=P["cci"], cci_mdf=P["cci_mdf"],
              mls=P["mls"], npt=npt, xg=g["gauss_x"] if len(g["gauss_x"]) else np.zeros(3 * n),
              gw=g["gw"] if len(g["gw"]) else np.array([2.0, 2.0, 2.0]),
              fam_ptr=g["fam_ptr"], fam_col=g["fam_col"], broken=g["broken"].astype(np.uint8),
              cb_ptr=g["cb_ptr"] if P["mls"] else None, cb_idx=g["cb_idx"] if P["mls"] else None,
              coeff=g["coeff"] if P["mls"] else None, bdry_eff=g["bdry_eff"], mat=g["mat"],
              mat_spring=g["spring"], mat_ecrit=g["mat_ecrit"], mat_density=g["mat_density"],
              mat_ymod=g["mat_ymod"], mat_grav=g["mat_grav"], bc=g["bc"], bc_type=g["bc_type"],
              bc_dir=g["bc_dir"], bc_val=g["bc_val"], bc_end=g["bc_end"], bc_load=g["bc_load"],
              damping=P["damping"])
    kw.update(over)
    return Model(**kw)
