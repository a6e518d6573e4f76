/*
 * Test infrastructure (oracle), not product code: a plain-C FP64 restatement
 * of empi's Matching Pursuit path.  Only tests/, the smoke check and bench.py's
 * CPU-baseline leg load it, as the checker.  See mp_oracle.c for the
 * reference file:line each function follows.
 */
#ifndef EMPI_MP_ORACLE_H
#define EMPI_MP_ORACLE_H

#ifdef __cplusplus
extern "C" {
#endif

typedef struct {
    double s;
    int nfft, fcount, tcount;
} or_scale;

/* variants, as in src/empi.cpp:114-130 */
enum { OR_SMP = 0, OR_MMP1 = 1, OR_MMP2 = 2, OR_MMP3 = 3 };

int or_geometry(double fs, int N, double energyError, double scaleMin, double scaleMax,
                double freqMax, int cap, or_scale* out);

int or_window_values(double fs, int N, double s, int nfft, int fcount, int tcount,
                     const double* x, int ti, double* values);

int or_energy_map(double fs, int C, int N, double energyError, double scaleMin, double scaleMax,
                  double freqMax, int mmp1, const double* samples, int scale, double* energy,
                  double* values);

int or_decompose(int variant, double fs, int C, int N, double energyError, double scaleMin,
                 double scaleMax, double freqMax, int iterationMax, double residualEnergy,
                 const double* samples, int maxAtoms, double* atoms, int* natoms, double* energies,
                 int* indices, double* margins, char* err, int errlen);

void or_subtract_atom(double* params, double* samples, int N, double fs, int fit);

#ifdef __cplusplus
}
#endif

#endif
