/* rn_oracle.h -- C-ABI of the CPU oracle (test infrastructure only).
 *
 * The oracle restates the reference's WebGL2 shader passes on the CPU; see the
 * header of rn_oracle.cpp. Only tests/, __graft_entry__.smoke() and bench.py's
 * CPU-baseline leg load it.
 */
#ifndef RN_ORACLE_H
#define RN_ORACLE_H
#include <stdint.h>
#ifdef __cplusplus
extern "C" {
#endif

/* The normalised parameter block P of the reference (simsetup.js:274-310) as
 * JavaScript doubles; the oracle rounds each to the arithmetic type the way
 * gl.uniform*fv rounds to float32. */
typedef struct {
  double amb[4], ambCons[4], ambB[4], gamR[2], inlet[4], res[3], gas[4], Rs[3], chemK[4], cap[2], chamberNu[2];
  double uInlet0, Tw, cfl, dtMax, wFloor, vMax, hllBlend, ramp, pStart, RcCells;
  int order2, inj, visc, chem;
  double mhat, tScale, fuelVec[4], oxVec[4], eF, eO, Ge;
} rno_params;

void* rno_create(int Nx, int Nr, int fp64);
void rno_destroy(void* h);
void rno_set_threads(int n);
void rno_set_geometry(void* h, const uint8_t* mask, const float* geoA, const float* geoG, const float* geoM,
                      const float* jWall);
void rno_set_state(void* h, const float* A, const float* B);
void rno_set_injector(void* h, const float* tab);
void rno_step(void* h, int n, const rno_params* p);
void rno_rescale_ambient(void* h, double fp, double fT, double du, const rno_params* p);
void rno_get_state(void* h, double* A, double* B);
void rno_get_step_info(void* h, double* out4);
void rno_get_wall_row(void* h, double* out);
void rno_get_t2(void* h, double* out);
void rno_set_parcels(void* h, const float* PA, const float* PB, int head);
void rno_get_parcels(void* h, double* PA, double* PB, double* PC);
void rno_get_spray_counters(void* h, uint32_t* head_seed);
void rno_get_src(void* h, double* out);

#ifdef __cplusplus
}
#endif
#endif
