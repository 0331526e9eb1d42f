/*
 * replay_ft -- the reference's finite-temperature driver, replayed in C
 * through the C ABI of libdqmc_gpu.so.
 *
 * The reference's main program (src/dqmc_main.f90:1-34) calls
 *   dqmc_initial; dqmc_start; dqmc_warmup;
 *   do nbc = 1, nbin: dqmc_sweep; dqmc_timing; end do
 *   dqmc_core_deallocate; dqmc_end
 * and dqmc_sweep (src/dqmc_ft_ctrl.f90:80-126) is
 *   obser_init; do nsw = 1, nsweep: sweep_b0(T,T); [ltau: push_stage,
 *   sweep_0b(F,F,T), pop_stage]; sweep_0b(T,T,F); end do; equaltime_output.
 * This program makes the same calls, in the same order, to the entry points
 * that replace them (include/dqmc_gpu.h), which is what the Fortran shim
 * include/dqmc_gpu_f.f90 does inside the reference.  It is a driver for hosts
 * without a Fortran compiler and the executable check of that call order.
 *
 * Usage: replay_ft [dqmc.in] [key=value ...]
 *   dqmc.in      the &model_para and &ctrl_para namelists (src/model_para.f90:155-218);
 *                keys la, lb, lc, beta, dtau, rt, rtd, t2, t3, nu, mu, rhub, rv, rhub_plq, alpha, theta,
 *                nflr, lproju, lprojv, lprojplqu, xmag, flux_x, flux_y, dimer, rndness,
 *                lstabilize, nwrap, nsweep, nbin, nublock, ltau, dyntau,
 *                obs_eqt_mid_len
 *   key=value    the same keys, plus the RUNMODE build flags of src/make.sys.*:
 *                lattice=1..5 (SQUARE|HONEYCOMB|CHAIN|CUBIC|R_CUBIC), update=0|1|2
 *                (fast|DELAY|SUBMATRIX), kinetic=0|1|2 (BREAKUP_T|FFT|zgemm),
 *                hs=0|1 (EXACTHS|general), and seed= (default: the -DTEST
 *                seed of rank 0, abs(2008*951049)), nwarmup= (default: nsweep
 *                on a fresh start, as dqmc_warmup; 0 under -DTEST), out=
 *                (default replay.out)
 * Output (out=): one line per bin, "bin nbc nobs" followed by the real and
 * imaginary parts of energy_bin(1:10) summed over the bin, then the
 * diagnostics of dqmc_end (src/dqmc_util.f90:287-299).  conf_u.in is read as
 * input_conf does (first integer /= 0: the field follows), and conf_u.out is
 * written at the end as dqmc_output_conf.
 */
#include <ctype.h>
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "../../include/dqmc_gpu.h"

static int g_fail = 0;
#define CALL(x)                                                                                    \
    do {                                                                                           \
        int rc_ = (x);                                                                             \
        if (rc_ != DQMC_OK) {                                                                      \
            fprintf(stderr, "replay_ft: %s returned %d: %s\n", #x, rc_, dqmc_gpu_last_error());    \
            g_fail = rc_;                                                                          \
            goto done;                                                                             \
        }                                                                                          \
    } while (0)

/* Fortran logical or number -> double */
static double fvalue(const char* s) {
    while (isspace((unsigned char)*s)) ++s;
    if (*s == '.') ++s;
    if (*s == 't' || *s == 'T') return 1.0;
    if (*s == 'f' || *s == 'F') return 0.0;
    char buf[64];
    size_t n = 0;
    for (; *s && n < sizeof(buf) - 1; ++s) buf[n++] = (*s == 'd' || *s == 'D') ? 'e' : *s;
    buf[n] = 0;
    return strtod(buf, NULL);
}

static int set_key(dqmc_params* p, const char* key, const char* val, int32_t* seed, int* nwarm, char* out) {
    char k[64];
    size_t n = 0;
    for (; key[n] && n < sizeof(k) - 1; ++n) k[n] = (char)tolower((unsigned char)key[n]);
    k[n] = 0;
    const double v = fvalue(val);
#define D(name) if (!strcmp(k, #name)) { p->name = v; return 0; }
#define I(name) if (!strcmp(k, #name)) { p->name = (int32_t)v; return 0; }
    if (!strcmp(k, "la")) { p->l1 = (int32_t)v; return 0; }
    if (!strcmp(k, "lb")) { p->l2 = (int32_t)v; return 0; }
    if (!strcmp(k, "lc")) { p->l3 = (int32_t)v; return 0; }
    if (!strcmp(k, "obs_eqt_mid_len")) { p->obs_mid_len = (int32_t)v; return 0; }
    if (!strcmp(k, "seed")) { *seed = (int32_t)v; return 0; }
    if (!strcmp(k, "nwarmup")) { *nwarm = (int)v; return 0; }
    if (!strcmp(k, "out")) { snprintf(out, 256, "%s", val); return 0; }
    D(beta) D(dtau) D(rt) D(t2) D(t3) D(nu) D(mu) D(rhub) D(rv) D(alpha) D(theta)
    D(xmag) D(flux_x) D(flux_y) D(dimer) D(rndness) D(dyntau) D(rtd) D(rhub_plq)
    I(l1) I(l2) I(nflr) I(lproju) I(lprojv) I(lprojplqu) I(lstabilize) I(nwrap) I(nsweep) I(nbin) I(nublock) I(ltau)
    I(lattice) I(update) I(kinetic) I(hs) I(proj)
#undef D
#undef I

    fprintf(stderr, "replay_ft: unknown key %s\n", key);
    return -1;
}

/* the entries of every &group ... / block: "key = value" separated by commas or newlines */
static int read_namelists(const char* path, dqmc_params* p, int32_t* seed, int* nwarm, char* out) {
    FILE* f = fopen(path, "r");
    if (!f) return 1;   /* no dqmc.in: defaults, as the reference */
    static char text[1 << 16];
    size_t n = fread(text, 1, sizeof(text) - 1, f);
    fclose(f);
    text[n] = 0;
    for (char* c = text; *c; ++c)   /* comments */
        if (*c == '!') while (*c && *c != '\n') *c++ = ' ';
    char* s = text;
    while ((s = strchr(s, '&')) != NULL) {
        while (*s && !isspace((unsigned char)*s)) ++s;   /* group name */
        char* end = strchr(s, '/');
        if (!end) end = s + strlen(s);
        char saved = *end;
        *end = 0;
        for (char* tok = strtok(s, ",\n"); tok; tok = strtok(NULL, ",\n")) {
            char* eq = strchr(tok, '=');
            if (!eq) continue;
            *eq = 0;
            char* key = tok;
            while (isspace((unsigned char)*key)) ++key;
            char* ke = key + strlen(key);
            while (ke > key && isspace((unsigned char)ke[-1])) *--ke = 0;
            if (*key && set_key(p, key, eq + 1, seed, nwarm, out)) return -1;
        }
        *end = saved;
        s = *end ? end + 1 : end;
    }
    return 0;
}

int main(int argc, char** argv) {
    dqmc_params p;
    memset(&p, 0, sizeof(p));
    /* defaults of src/model_para.f90:166-206 and the square Hubbard build */
    p.lattice = DQMC_LATT_SQUARE; p.l1 = 2; p.l2 = 2; p.l3 = 2; p.rtd = 1.0; p.beta = 20.0; p.dtau = 0.05; p.rt = 1.0;
    p.alpha = 0.2; p.nflr = 2; p.lstabilize = 1; p.nwrap = 10; p.nsweep = 20; p.nbin = 10;
    p.update = DQMC_UPD_DELAY; p.kinetic = DQMC_KIN_CHECKERBOARD; p.hs = DQMC_HS_GENERAL4; p.obs_mid_len = 1;
    int32_t seed = 1909706392;   /* abs((0*1981+2008)*951049), src/dqmc_util.f90:72 under -DTEST */
    int nwarm = -1;
    char out[256] = "replay.out";
    int a0 = 1;
    if (argc > 1 && !strchr(argv[1], '=')) {
        if (read_namelists(argv[1], &p, &seed, &nwarm, out) < 0) return 2;
        a0 = 2;
    }
    for (int a = a0; a < argc; ++a) {
        char* eq = strchr(argv[a], '=');
        if (!eq) { fprintf(stderr, "replay_ft: argument %s is not key=value\n", argv[a]); return 2; }
        *eq = 0;
        if (set_key(&p, argv[a], eq + 1, &seed, &nwarm, out)) return 2;
    }

    dqmc_handle* h = NULL;
    FILE* fo = NULL;
    int32_t* conf = NULL;
    double* bins = NULL;
    /* dqmc_initial: make_tables (src/model_para.f90:334-453) */
    CALL(dqmc_params_derive(&p));
    const int N = p.ndim, lt = p.ltrot;
    conf = (int32_t*)malloc(sizeof(int32_t) * (size_t)N * lt);
    /* dqmc_start: set_h0conf, set_conf, input_conf (a fresh start draws the field), allocate_core */
    CALL(dqmc_gpu_create(&p, 1, 1, &seed, 1, &h));
    int fresh = 1;
    {
        FILE* fc = fopen("conf_u.in", "r");
        int flag = 0;
        if (fc && fscanf(fc, "%d", &flag) == 1 && flag != 0) {
            /* input_conf (src/dqmc_config_u/dqmc_input_conf.f90:21-54): the rank-0 block */
            int ok = 1;
            for (size_t e = 0; e < (size_t)N * lt && ok; ++e) ok = fscanf(fc, "%d", &conf[e]) == 1;
            if (!ok) { fprintf(stderr, "replay_ft: conf_u.in is short\n"); fclose(fc); g_fail = 2; goto done; }
            CALL(dqmc_gpu_set_conf(h, 0, conf));
            fresh = 0;
        }
        if (fc) fclose(fc);
    }
    CALL(dqmc_gpu_sweep_start(h));
    /* dqmc_warmup (src/dqmc_ft_ctrl.f90:52-78): nsweep warm-up sweeps on a fresh start */
    if (nwarm < 0) nwarm = fresh ? p.nsweep : 0;
    for (int i = 0; i < nwarm; ++i) {
        CALL(dqmc_gpu_sweep_b0(h, 1, 0));
        CALL(dqmc_gpu_sweep_0b(h, 1, 0));
    }
    fo = fopen(out, "w");
    if (!fo) { fprintf(stderr, "replay_ft: cannot write %s\n", out); g_fail = 2; goto done; }
    bins = (double*)malloc(sizeof(double) * 2 * 20);
    for (int nbc = 1; nbc <= p.nbin; ++nbc) {
        /* dqmc_sweep */
        CALL(dqmc_gpu_obser_init(h));
        for (int nsw = 1; nsw <= p.nsweep; ++nsw) {
            CALL(dqmc_gpu_sweep_b0(h, 1, 1));
            if (p.ltau) CALL(dqmc_gpu_sweep_dyn(h));
            CALL(dqmc_gpu_sweep_0b(h, 1, 1));
        }
        /* equaltime_output: the bin sums (the energy block leads the layout) */
        int nb = dqmc_gpu_nbins(h, 0);
        if (nb < 10) { fprintf(stderr, "replay_ft: dqmc_gpu_nbins returned %d\n", nb); g_fail = 2; goto done; }
        double* all = (double*)malloc(sizeof(double) * 2 * (size_t)nb);
        int rc = dqmc_gpu_get_bins(h, 0, all);
        if (rc) { free(all); CALL(rc); }
        memcpy(bins, all, sizeof(double) * 20);
        free(all);
        dqmc_diag d;
        CALL(dqmc_gpu_get_diag(h, 0, &d));
        fprintf(fo, "bin %d %.0f", nbc, d.nobs);
        for (int k = 0; k < 10; ++k) fprintf(fo, " %.17e %.17e", bins[2 * k], bins[2 * k + 1]);
        fprintf(fo, "\n");
        /* dqmc_timing: dqmc_output_conf */
        CALL(dqmc_gpu_get_conf(h, 0, conf));
    }
    {
        /* dqmc_end (src/dqmc_util.f90:287-299) */
        dqmc_diag d;
        CALL(dqmc_gpu_get_diag(h, 0, &d));
        fprintf(fo, "max_wrap_error %.8e\n", d.max_wrap_error);
        fprintf(fo, "max_phasediff %.8e\n", d.max_phasediff);
        fprintf(fo, "accep_u %.8e\n", d.proposed > 0 ? d.accepted / d.proposed : 0.0);
        FILE* fc = fopen("conf_u.out", "w");
        if (fc) {   /* dqmc_output_conf (src/dqmc_config_u/dqmc_output_conf.f90:27-42) */
            fprintf(fc, "%12d\n", 1);
            for (size_t e = 0; e < (size_t)N * lt; ++e) fprintf(fc, "%4d\n", conf[e]);
            fclose(fc);
        }
    }
done:
    if (fo) fclose(fo);
    free(conf);
    free(bins);
    if (h) dqmc_gpu_destroy(h);
    return g_fail ? 1 : 0;
}
