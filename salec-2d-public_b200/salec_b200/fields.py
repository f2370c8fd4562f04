"""Field sets of the device state, by the reference's member names of sale2d_var."""

# every field the step reads or writes (the state to upload when handing a run to the device)
STEP_FIELDS = [
    "v_vel", "v_bf", "v_acc", "v_dis", "v_pos", "v_vof", "v_mass", "v_vol", "v_subvol", "v_laplace", "v_suf",
    "v_alpha", "e_vel", "e_div_vel", "e_grad_vel", "e_ste", "e_mu", "e_dvel", "e_pre", "e_tem", "e_den", "e_csd",
    "e_dam", "e_cvs", "m_vof", "m_den", "m_eng", "m_pty", "e_wpt", "e_pos", "e_vol", "e_grad", "e_q",
    "e_strength", "e_cnd", "e_tps", "e_ste2s", "e_sta2s", "e_alpha", "e_beta", "e_sigma", "e_dampref", "e_vib",
    "e_ejt", "bx_phi", "by_phi", "bx_normal", "by_normal", "y_profile",
]

# fields the step evolves
STATE_FIELDS = [
    "v_vel", "v_acc", "v_dis", "v_vof", "v_mass", "v_alpha", "e_vel", "e_div_vel", "e_grad_vel", "e_ste", "e_mu",
    "e_dvel", "e_pre", "e_tem", "e_den", "e_csd", "e_dam", "e_cvs", "m_vof", "m_den", "m_eng", "m_pty", "e_wpt",
    "e_q", "e_strength", "e_tps", "e_ste2s", "e_sta2s", "e_alpha", "e_beta", "e_vib", "e_ejt", "e_cnd", "y_profile",
]

# fields the reference writes to its VTS files at an output cycle (src/write_vtk.c:253-298)
OUTPUT_FIELDS = [
    "v_vel", "v_acc", "v_bf", "v_vof", "e_den", "e_pre", "e_wpt", "m_vof", "e_csd", "e_dam", "e_tps", "e_q",
    "e_tem", "m_eng", "m_den", "e_ste2s", "e_sta2s", "e_ste", "e_strength", "e_vib", "e_ejt", "e_cvs", "m_pty",
    "v_pos",
]
