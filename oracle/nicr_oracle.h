/* Test infrastructure only (the oracle): a plain-C restatement of the
 * reference's explicit time step and its initialisation, run on the CPU to
 * check the CUDA path. Only tests/, __graft_entry__.smoke() and bench.py's
 * CPU-baseline leg may load it; the product never does. */
#ifndef NICR_ORACLE_H
#define NICR_ORACLE_H
#include "../include/nicr.h"

typedef struct omodel omodel;

omodel* oracle_create(const nicr_config* cfg, char* err, int errlen);
void oracle_destroy(omodel* m);
long long oracle_ncells(const omodel* m);
int oracle_neta(const omodel* m);
int oracle_nseeds(const omodel* m);
int oracle_center_seed_cells(const omodel* m);
/* name: o cr p muO muCr mo mc gb grain eta_s2 eta_pairs gb_initial etaN (N 1-based) */
int oracle_get(omodel* m, const char* name, double* out);
int oracle_set_fields(omodel* m, const double* o, const double* cr, const double* p, const double* eta);
void oracle_reset_inventory(omodel* m);
void oracle_refresh(omodel* m);
void oracle_invalidate(omodel* m);
int oracle_step(omodel* m);                       /* 0 ok, else NICR_ERR_* */
int oracle_run(omodel* m, int steps, int* done);  /* run() schedule        */
void oracle_nucleate(omodel* m);
int oracle_stamp(omodel* m, int x, int y, int z);
int oracle_scale_eta(omodel* m, int g, int i, int j, int k, double f);
const char* oracle_error(const omodel* m);
/* budget: nucO nucCr ckO ckCr clipO clipCr bcO bcCr initialO initialCr as hi,lo pairs (20 doubles) */
void oracle_budget(const omodel* m, double* hilo, long long* counts);
void oracle_seeds(const omodel* m, double* xyz, long long* volumes);
/* log row values: so sc po(sum) sumH as hi,lo pairs (8) then omin omax crmin crmax nimin phimin phimax (7) */
void oracle_log_values(omodel* m, double* out);
/* grain row: lo hi slo shi, sumS(hi,lo), mask(hi,lo), energy(hi,lo), gbmax, alive, unassigned;
 * cells[neta], amount[2*neta] (hi,lo) */
int oracle_grain_values(omodel* m, double* out, long long* cells, double* amount);
#endif
