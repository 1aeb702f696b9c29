// Golden-vector generator (test infrastructure): a driver linked against the
// reference's own FP32 scalar build (oracle/_ref/libcgfdm_ref_fp32.so) that
// runs the reference's setup and one RK stage of its hot path and dumps the
// results as raw float32 files in the working directory.
//
//   ref_dump setup                 -> setup_*.bin (incl. the scaled finite-fault
//                                     moment rates when useMultiSource is set)
//   ref_dump stage IRK FB1 FB2 FB3 -> reads in_*.bin, writes out_*.bin
//
// The sequence of calls mirrors run.cpp:56-111 (setup) and propagate.cpp:
// 157-167 (one stage, single rank: every MPI border present).
#include "header.h"

static void dump(const char *name, const void *p, size_t bytes) {
  FILE *f = fopen(name, "wb");
  fwrite(p, 1, bytes, f);
  fclose(f);
}
static void load(const char *name, void *p, size_t bytes) {
  FILE *f = fopen(name, "rb");
  if (!f || fread(p, 1, bytes, f) != bytes) {
    fprintf(stderr, "ref_dump: cannot read %s\n", name);
    exit(2);
  }
  fclose(f);
}

int main(int argc, char **argv) {
  if (argc < 2) return 2;
  PARAMS params;
  memset(&params, 0, sizeof params);
  GRID grid = {0};
  MPI_COORD coord3 = {0};
  MPI_NEIGHBOR nb = {0};
  MPI_Comm comm;
  getParams(&params);
  init_MPI(&argc, &argv, params, &comm, &coord3, &nb);
  init_grid(params, &grid, coord3);
  createDir(params);

  float *coord, *cpu_coord, *terrain, *cpu_terrain, *medium, *cpu_medium;
  allocTerrain(grid, &terrain, &cpu_terrain);
  allocCoord(grid, &coord, &cpu_coord);
  constructCoord(comm, coord3, grid, params, coord, cpu_coord, terrain, cpu_terrain);
  allocMedium(grid, &medium, &cpu_medium);
  constructMedium(coord3, params, grid, cpu_coord, cpu_terrain, medium, cpu_medium);
  long long num = (long long)grid._nx_ * grid._ny_ * grid._nz_;
  long long nsurf = (long long)grid._nx_ * grid._ny_;
  dump("setup_coord.bin", cpu_coord, sizeof(float) * num * CSIZE);
  dump("setup_medium.bin", cpu_medium, sizeof(float) * num * MSIZE);
  dump("setup_terrain.bin", cpu_terrain, sizeof(float) * nsurf);

  FLOAT *CJM;
  allocCJM(grid, &CJM);
  Mat_rDZ rdz;
  allocMat_rDZ(grid, &rdz);
  constructCJM(comm, nb, grid, CJM, coord, medium, rdz);
  dump("setup_cjm.bin", CJM, sizeof(FLOAT) * num * CJMSIZE);
  dump("setup_rdz.bin", rdz._rDZ_DX, sizeof(float) * nsurf * 2 * MATSIZE);

  MPI_BORDER border = {1, 1, 1, 1, 1, 1};
  PML_ALPHA pa;
  PML_BETA pb;
  PML_D pd;
  allocPMLParameter(grid, &pa, &pb, &pd);
  init_pml_parameter(params, grid, border, pa, pb, pd);
  dump("setup_pml.bin", pa.x, sizeof(float) * (grid._nx_ + grid._ny_ + grid._nz_) * 3);

  if (params.useMultiSource) {  // run.cpp:123-127 then propagate.cpp:124-128
    long long *srcIndex = NULL;
    float *momentRate = NULL, *momentRateSlice = NULL;
    SOURCE_FILE_INPUT src_in;
    init_MultiSource(params, grid, coord3, cpu_coord, cpu_terrain, &srcIndex, &momentRate,
                     &momentRateSlice, &src_in);
    calculateMomentRate(src_in, CJM, momentRate, srcIndex, grid);
    int hdr[2] = {(int)src_in.npts, src_in.nt};
    dump("setup_src_hdr.bin", hdr, sizeof hdr);
    dump("setup_src_index.bin", srcIndex, sizeof(long long) * src_in.npts);
    dump("setup_src_rate.bin", momentRate, sizeof(float) * src_in.npts * src_in.nt * MOMSIZE);
  }

  if (!strcmp(argv[1], "stage") && argc >= 6) {
    int irk = atoi(argv[2]), FB1 = atoi(argv[3]), FB2 = atoi(argv[4]), FB3 = atoi(argv[5]);
    float DT = params.DT;
    WAVE wave;
    allocWave(grid, &wave);
    load("in_W.bin", wave.W, sizeof(FLOAT) * num * WSIZE);
    load("in_t.bin", wave.t_W, sizeof(FLOAT) * num * WSIZE);
    load("in_m.bin", wave.m_W, sizeof(FLOAT) * num * WSIZE);
    AUX6SURF aux;
    allocPML(grid, &aux, border);
    AUX *slabs[5] = {&aux.Aux1x, &aux.Aux1y, &aux.Aux1z, &aux.Aux2x, &aux.Aux2y};
    long long npos[5] = {
        (long long)grid.nPML * grid.ny * grid.nz, (long long)grid.nx * grid.nPML * grid.nz,
        (long long)grid.nx * grid.ny * grid.nPML, (long long)grid.nPML * grid.ny * grid.nz,
        (long long)grid.nx * grid.nPML * grid.nz};
    FILE *fa = fopen("in_aux.bin", "rb");
    for (int s = 0; s < 5; ++s) {
      size_t b = sizeof(float) * npos[s] * WSIZE;
      if (fread(slabs[s]->Aux, 1, b, fa) != b || fread(slabs[s]->t_Aux, 1, b, fa) != b ||
          fread(slabs[s]->m_Aux, 1, b, fa) != b) {
        fprintf(stderr, "ref_dump: short in_aux.bin\n");
        return 2;
      }
    }
    fclose(fa);

    waveDeriv(grid, wave, CJM, pb, FB1, FB2, FB3, DT);
    freeSurfaceDeriv(grid, wave, CJM, rdz, pb, FB1, FB2, FB3, DT);
    pmlDeriv(grid, wave, CJM, aux, pa, pb, pd, border, FB1, FB2, FB3, DT);
    pmlFreeSurfaceDeriv(grid, wave, CJM, aux, rdz, pd, border, FB1, FB2, DT);
    dump("out_h.bin", wave.h_W, sizeof(FLOAT) * num * WSIZE);
    waveRk(grid, irk, wave);
    pmlRk(grid, border, irk, aux);
    dump("out_W.bin", wave.W, sizeof(FLOAT) * num * WSIZE);
    dump("out_t.bin", wave.t_W, sizeof(FLOAT) * num * WSIZE);
    dump("out_m.bin", wave.m_W, sizeof(FLOAT) * num * WSIZE);
    fa = fopen("out_aux.bin", "wb");
    for (int s = 0; s < 5; ++s) {
      size_t b = sizeof(float) * npos[s] * WSIZE;
      fwrite(slabs[s]->h_Aux, 1, b, fa);
      fwrite(slabs[s]->Aux, 1, b, fa);
      fwrite(slabs[s]->t_Aux, 1, b, fa);
      fwrite(slabs[s]->m_Aux, 1, b, fa);
    }
    fclose(fa);
  }
  MPI_Finalize();
  return 0;
}
