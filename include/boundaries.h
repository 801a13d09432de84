/* boundaries.h -- boundary collision rules of the drop-in interface (liblbgpu.so).
 *
 * Source-compatible with the reference's boundaries.h: the two parameter blocks and the 17
 * boundary functions with the same prototypes (reference boundaries.h:50-102).  Each
 * function is a working host implementation with the reference's arithmetic (drivers may
 * call them on a single node), and its address is what tells the GPU library which rule a
 * node follows.  On the device every rule chains to bulk BGK, so `bulkDynamics` must be a
 * Dynamics whose function is bgk.
 */
#ifndef BOUNDARIES_H
#define BOUNDARIES_H

#include "lb.h"

#ifdef __cplusplus
extern "C" {
#endif

/* Prescribed velocity on a straight wall (reference boundaries.h:50-53). */
typedef struct {
    Dynamics *bulkDynamics;
    double ux, uy;
} VelocityBCData;

/* Prescribed density and tangential velocity (reference boundaries.h:64-67). */
typedef struct {
    Dynamics *bulkDynamics;
    double rho, uPar;
} PressureBCData;

/* Full-way bounce-back; selfData unused (reference boundaries.h:74). */
void bounceBack(double *fPop, void *selfData);

/* Zou/He velocity and pressure rules (reference boundaries.h:78-88). */
void upperZouHe(double *fPop, void *selfData);
void lowerZouHe(double *fPop, void *selfData);
void leftZouHe(double *fPop, void *selfData);
void rightZouHe(double *fPop, void *selfData);
void upperPressureZouHe(double *fPop, void *selfData);
void lowerPressureZouHe(double *fPop, void *selfData);
void leftPressureZouHe(double *fPop, void *selfData);
void rightPressureZouHe(double *fPop, void *selfData);

/* Regularized velocity and pressure rules (reference boundaries.h:92-102). */
void upperRegularized(double *fPop, void *selfData);
void lowerRegularized(double *fPop, void *selfData);
void leftRegularized(double *fPop, void *selfData);
void rightRegularized(double *fPop, void *selfData);
void upperPressureRegularized(double *fPop, void *selfData);
void lowerPressureRegularized(double *fPop, void *selfData);
void leftPressureRegularized(double *fPop, void *selfData);
void rightPressureRegularized(double *fPop, void *selfData);

#ifdef __cplusplus
}
#endif
#endif
