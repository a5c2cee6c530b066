/*
 * Prints the size and field offsets of the structs the CUDA-backend C-ABI
 * passes by pointer (FcaPhys, FcaRunCfg, FcaComm, FcaGrid, FcaAcc, FcaTimers)
 * as one JSON object. Test infrastructure: compiled once against the
 * reference's src/common/fca_types.h (oracle/Makefile.ref) to make the layout
 * fixture, and once against include/floodca_b200.h by the CPU tests, which
 * compare the two.
 */
#include <stddef.h>
#include <stdio.h>

#ifdef PROBE_OWN_HEADER
#include "floodca_b200.h"
#else
#include "fca_types.h"
#endif

static int first = 1;

static void sz(const char *s, size_t v)
{
    printf("%s\"%s\": %zu", first ? "" : ",\n", s, v);
    first = 0;
}

#define F(T, f) sz(#T "." #f, offsetof(T, f))
#define S(T) sz("sizeof(" #T ")", sizeof(T))

int main(void)
{
    printf("{\n");
    S(real);
    S(FcaPhys);
    F(FcaPhys, dx); F(FcaPhys, A); F(FcaPhys, g); F(FcaPhys, alpha); F(FcaPhys, tau_h);
    F(FcaPhys, tau_l); F(FcaPhys, z_sea); F(FcaPhys, dt_max); F(FcaPhys, dt_min);
    F(FcaPhys, S_bnd); F(FcaPhys, h_flood); F(FcaPhys, U); F(FcaPhys, K); F(FcaPhys, boundary);
    S(FcaRunCfg);
    F(FcaRunCfg, phys); F(FcaRunCfg, T_sim); F(FcaRunCfg, out_every); F(FcaRunCfg, diag_every);
    F(FcaRunCfg, progress_every); F(FcaRunCfg, hyeto); F(FcaRunCfg, D_h); F(FcaRunCfg, phi);
    F(FcaRunCfg, lambda); F(FcaRunCfg, steps); F(FcaRunCfg, no_output); F(FcaRunCfg, neigh);
    F(FcaRunCfg, config_path); F(FcaRunCfg, grid_dir); F(FcaRunCfg, scenario);
    F(FcaRunCfg, scenario_file); F(FcaRunCfg, warmstart); F(FcaRunCfg, rain_file);
    F(FcaRunCfg, out_dir); F(FcaRunCfg, csv_path); F(FcaRunCfg, exp_id); F(FcaRunCfg, repeat);
    F(FcaRunCfg, threads); F(FcaRunCfg, ranks); F(FcaRunCfg, gpus); F(FcaRunCfg, block_x);
    F(FcaRunCfg, block_y); F(FcaRunCfg, halo_mode); F(FcaRunCfg, reduce_impl);
    F(FcaRunCfg, gpu_model); F(FcaRunCfg, backend); F(FcaRunCfg, forcing_csv);
    F(FcaRunCfg, n_force_days); F(FcaRunCfg, force_files);
    S(FcaComm);
    F(FcaComm, ctx); F(FcaComm, rank); F(FcaComm, halo); F(FcaComm, min_real);
    F(FcaComm, sum_double); F(FcaComm, load_rday);
    S(FcaGrid);
    F(FcaGrid, nrows); F(FcaGrid, ncols); F(FcaGrid, r0); F(FcaGrid, r1); F(FcaGrid, c0);
    F(FcaGrid, c1); F(FcaGrid, edge_n); F(FcaGrid, edge_s); F(FcaGrid, edge_w);
    F(FcaGrid, edge_e); F(FcaGrid, comm); F(FcaGrid, dx); F(FcaGrid, x0); F(FcaGrid, y0);
    F(FcaGrid, z); F(FcaGrid, h); F(FcaGrid, n); F(FcaGrid, C); F(FcaGrid, mask);
    F(FcaGrid, Rday); F(FcaGrid, hmax); F(FcaGrid, tmax); F(FcaGrid, s); F(FcaGrid, out);
    F(FcaGrid, Qx); F(FcaGrid, Qy); F(FcaGrid, Qd1); F(FcaGrid, Qd2); F(FcaGrid, Qopen);
    S(FcaAcc);
    F(FcaAcc, V); F(FcaAcc, V0); F(FcaAcc, V_rain); F(FcaAcc, V_sea); F(FcaAcc, V_bnd);
    F(FcaAcc, clamp_err); F(FcaAcc, cap_active); F(FcaAcc, cap_total); F(FcaAcc, dt_min_hits);
    F(FcaAcc, t); F(FcaAcc, step); F(FcaAcc, dt_base); F(FcaAcc, force_day);
    S(FcaTimers);
    F(FcaTimers, wall_total); F(FcaTimers, t_init); F(FcaTimers, t_flux);
    F(FcaTimers, t_limiter); F(FcaTimers, t_update); F(FcaTimers, t_dt); F(FcaTimers, t_io);
    F(FcaTimers, t_h2d); F(FcaTimers, t_d2h); F(FcaTimers, t_halo); F(FcaTimers, t_allreduce);
    F(FcaTimers, bytes_per_step); F(FcaTimers, active_cells);
    printf("\n}\n");
    return 0;
}
