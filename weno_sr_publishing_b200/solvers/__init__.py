"""Adapters with the reference's solver call signatures (allocate_forward, launch_stage, advance_step,
run_to_time) for WENO5-JS (weno5_hllc), WENO5-SR with an FP64 closure (weno5_hllc_refsym) and WENO5-SR
with an FP32 closure (weno5_hllc_mixed), and WENO5-Z with eps = h^2 (weno5_hllc_z_min, and
weno5_double_mach_z on the double-Mach boundary). Boundaries: "transmissive", "periodic", "double-mach"."""
