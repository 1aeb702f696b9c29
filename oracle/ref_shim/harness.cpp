/*
 * Test infrastructure (oracle harness), not product code.
 *
 * Link-time replacements for the three reference functions that need data or
 * libraries that are not available here (PROJ, SRTM90 DEM tiles, the Shen and
 * CRUST1.0 model directories).  Everything else of the reference is compiled
 * unchanged from its own sources.
 *
 *  - preprocessTerrain (src-new-FP32-SVE/terrain.cpp:839-940): instead of
 *    interpolating DEM tiles, the terrain height h(I,J) of the whole padded
 *    grid is read from "terrain_input.bin" in the working directory
 *    (float32, (NY+6) rows of (NX+6) values, x fastest).  The rank's part is
 *    cut out and the reference's own vertical stretch is applied
 *    (terrain.cpp:917-937: z = -|Depth| + (h+|Depth|)/(NZ-1) * K).
 *    The SRTM90 build (make ref-srtm, -DCGFDM_HARNESS_REF_TERRAIN) keeps the
 *    reference's own preprocessTerrain instead.
 *  - readWeisenShenModel / readCrustal_1: not used by any fixture; they abort.
 */
#include "header.h"

#ifndef CGFDM_HARNESS_REF_TERRAIN
void preprocessTerrain(PARAMS params, MPI_Comm comm_cart, MPI_COORD thisMPICoord, GRID grid,
                       float *coord, float *terrain) {
  (void)comm_cart;
  (void)thisMPICoord;
  const int halo = grid.halo;
  const int _nx_ = grid._nx_, _ny_ = grid._ny_, _nz_ = grid._nz_;
  const int NXP = grid.NX + 2 * HALO, NYP = grid.NY + 2 * HALO;

  FILE *fp = fopen("terrain_input.bin", "rb");
  if (!fp) {
    printf("harness: terrain_input.bin is missing\n");
    MPI_Abort(MPI_COMM_WORLD, 100);
  }
  float *global = (float *)malloc(sizeof(float) * (size_t)NXP * NYP);
  size_t got = fread(global, sizeof(float), (size_t)NXP * NYP, fp);
  fclose(fp);
  if (got != (size_t)NXP * NYP) {
    printf("harness: terrain_input.bin holds %zu values, expected %d\n", got, NXP * NYP);
    MPI_Abort(MPI_COMM_WORLD, 100);
  }
  for (int j = 0; j < _ny_; ++j)
    for (int i = 0; i < _nx_; ++i)
      terrain[Index2D(i, j, _nx_, _ny_)] =
          global[(size_t)(grid.frontNX + i) + (size_t)(grid.frontNY + j) * NXP];
  free(global);

  double Depth = params.Depth * 1e3;
  int NZ = grid.NZ;
  int frontNZ = grid.frontNZ;
  for (int k = 0; k < _nz_; ++k)
    for (int j = 0; j < _ny_; ++j)
      for (int i = 0; i < _nx_; ++i) {
        long long index = INDEX(i, j, k) * CSIZE;
        int pos = Index2D(i, j, _nx_, _ny_);
        int K = frontNZ + k - halo;
        double DZ = double(terrain[pos] + abs(Depth)) / double(NZ - 1);
        coord[index + 2] = -abs(Depth) + DZ * K;
      }
}
#endif  // the SRTM90 build (make ref-srtm) compiles the reference's own terrain.cpp

void readWeisenShenModel(PARAMS, GRID, MPI_COORD, float *, float *, float *) {
  printf("harness: the Shen crust model is not available\n");
  MPI_Abort(MPI_COMM_WORLD, 100);
}

void readCrustal_1(PARAMS, GRID, MPI_COORD, float *, float *) {
  printf("harness: the CRUST1.0 model is not available\n");
  MPI_Abort(MPI_COMM_WORLD, 100);
}
