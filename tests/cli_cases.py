"""Command lines of the calllmie fixtures (tests/golden/cli/<name>/): each is
run by the reference's calllmie when the fixtures are made and by
lmie_b200/calllmie in tests/test_cli.py, in a directory of its own, so the
output file names are relative."""

CLI_CASES = {
    # every output kind and both self-checks, no derivatives
    "lognormal_all": [
        "-dist", "log_normal", "0.1", "0.164402", "0.005", "2.0", "-lambda", "0.55", "-m", "1.45", "0.001",
        "-n_int2", "1", "-n_quad", "200", "-n_angles", "181", "-total", "-", "-gc", "gc.txt", "-lc", "lc.txt",
        "-pf", "pf.txt", "-check_cbak", "1e-5", "-check_g", "1e-5"],
    # four derivatives (mr, mi, a1, a2), one file per derivative
    "gamma_derivs": [
        "-derivs", "4", "-dist", "gamma", "2.0", "0.1", "0.01", "6.0", "-dist_l", "0,0,1,0", "0,0,0,1",
        "0,0,0,0", "0,0,0,0", "-lambda", "0.865", "-m", "1.335", "1e-6", "-m_l", "1,0,0,0", "0,1,0,0",
        "-n_int2", "2", "-n_quad", "100", "-n_angles", "91",
        "-total", "total.txt", "t_mr.txt,t_mi.txt,t_a1.txt,t_a2.txt",
        "-gc", "gc.txt", "gc_mr.txt,gc_mi.txt,gc_a1.txt,gc_a2.txt",
        "-pf", "pf.txt", "pf_mr.txt,pf_mi.txt,pf_a1.txt,pf_a2.txt"],
    # one radius, solved again from the saved per-radius quantities
    "mono_save": [
        "-dist", "mono", "1.0", "-lambda", "0.6", "-m", "1.5", "0.01", "-n_int2", "1", "-n_quad", "1",
        "-n_angles", "61", "-save_dist", "-gc", "gc.txt", "-pf", "pf.txt", "-total", "-"],
}
