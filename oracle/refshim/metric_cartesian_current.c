/*
 * TEST INFRASTRUCTURE ONLY.
 *
 * The reference's metrics/metric_cartesian.c no longer compiles against its own
 * decs.h (r_of_x/th_of_x signatures, decs.h:1011-1012; it indexes geom with ND_ELEM
 * where the collapsed allocation needs ND_ELEM_LINEAR).  This file restates the same
 * trivial Cartesian metric (metric_cartesian.c:47-295) in the current API so that the
 * rest of the reference hydro can be built unmodified around it:
 *   alpha0 = (x1^3-x0^3)/3, beta0 = (x1^2-x0^2)/2, Gamma0 = dx   (metric_cartesian.c:47-55)
 *   volume = prod dx, area[l] = prod dx / dx[l], gcov = gcon = scale = 1, conn = 0.
 */
#include "decs.h"

void init_coords() { return; }

void ijk_to_x(int i, int j, int k, double x[SPACEDIM])
{
  int dd;
  int index[] = {i, j, k};
  DLOOP { x[dd] = (index[dd]+0.5)*dx[dd] + startx[dd]; }
}

void x_to_ijk(double x[], int index[])
{
  int dd;
  DLOOP { index[dd] = (x[dd]-startx[dd])/dx[dd]; }
}

void ijk_to_Cart(int i, int j, int k, double *x)
{
  x[0] = startx[0] + i*dx[0];
#if (NDIM>1)
  x[1] = startx[1] + j*dx[1];
#endif
#if (NDIM==3)
  x[2] = startx[2] + k*dx[2];
#endif
}

double ijk_to_r(int i, int j, int k, double *rhat)
{
  int dd;
  double x[SPACEDIM], r = 0.0;
  ijk_to_x(i,j,k,x);
  DLOOP { r += SQR(x[dd]); }
  r = sqrt(r);
  DLOOP { rhat[dd] = x[dd]/r; }
  return r;
}

void init_interp_vol()
{
  int i;
  double x0, x1;
  for (i=istart[0]-NG; i<istop[0]+NG; i++) {
    x0 = startx[0] + i*dx[0];
    x1 = x0 + dx[0];
    alpha0[i] = (CUBE(x1) - CUBE(x0))/3.0;
    beta0[i]  = (SQR(x1) - SQR(x0))/2.0;
    Gamma0[i] = dx[0];
  }
#if (NDIM>1)
  {
    int j, n2s = global_grid_dims[1] + 2*NG;
    Gamma1s = malloc_rank1(1, sizeof *Gamma1s);
    beta1s  = malloc_rank1(1, sizeof *beta1s );
    alpha1s = malloc_rank1(1, sizeof *alpha1s);
    Gamma1s[0] = (double*)malloc_rank1(n2s, sizeof *Gamma1s[0]) + NG - istart[1];
    beta1s [0] = (double*)malloc_rank1(n2s, sizeof *beta1s [0]) + NG - istart[1];
    alpha1s[0] = (double*)malloc_rank1(n2s, sizeof *alpha1s[0]) + NG - istart[1];
    for (j=istart[1]-NG; j<istop[1]+NG; j++) {
      x0 = startx[1] + j*dx[1];
      x1 = x0 + dx[1];
      alpha1s[0][j] = (CUBE(x1) - CUBE(x0))/3.0;
      beta1s[0][j]  = (SQR(x1) - SQR(x0))/2.0;
      Gamma1s[0][j] = dx[1];
    }
  }
#endif
#if (NDIM==3)
  {
    int k, n3s = global_grid_dims[2] + 2*NG;
    Gamma2s = malloc_rank1(1, sizeof *Gamma2s);
    beta2s  = malloc_rank1(1, sizeof *beta2s );
    alpha2s = malloc_rank1(1, sizeof *alpha2s);
    Gamma2s[0] = (double*)malloc_rank1(n3s, sizeof *Gamma2s[0]) + NG - istart[2];
    beta2s [0] = (double*)malloc_rank1(n3s, sizeof *beta2s [0]) + NG - istart[2];
    alpha2s[0] = (double*)malloc_rank1(n3s, sizeof *alpha2s[0]) + NG - istart[2];
    for (k=istart[2]-NG; k<istop[2]+NG; k++) {
      x0 = startx[2] + k*dx[2];
      x1 = x0 + dx[2];
      alpha2s[0][k] = (CUBE(x1) - CUBE(x0))/3.0;
      beta2s[0][k]  = (SQR(x1) - SQR(x0))/2.0;
      Gamma2s[0][k] = dx[2];
    }
  }
#endif
}

void calc_interp_coeffs1(int i, double *alpha, double *beta, double *Gamma, double *x)
{
#if (NDIM>1)
  for (int j=istart[1]-NG; j<istop[1]+NG; j++) {
    alpha[j-istart[1]] = alpha1s[0][j];
    beta[j-istart[1]] = beta1s[0][j];
    Gamma[j-istart[1]] = Gamma1s[0][j];
    x[j-istart[1]] = startx[1] + j*dx[1];
  }
#endif
}

void calc_interp_coeffs2(int i, int j, double *alpha, double *beta, double *Gamma, double *x)
{
#if (NDIM==3)
  for (int k=istart[2]-NG; k<istop[2]+NG; k++) {
    alpha[k-istart[2]] = alpha2s[0][k];
    beta[k-istart[2]] = beta2s[0][k];
    Gamma[k-istart[2]] = Gamma2s[0][k];
    x[k-istart[2]] = startx[2] + k*dx[2];
  }
#endif
}

void vec_transform_to_xyz(double *vp, int i, int j, int k) { return; }

/* zone loops over all cells including the ghost corners (ZGLOOP) */
void init_volume()
{
  int ii=0, jj=0, kk=0, dd;
  ZGLOOP {
    ND_ELEM_LINEAR(geom,ii,jj,kk).volume = 1.0;
    DLOOP { ND_ELEM_LINEAR(geom,ii,jj,kk).volume *= dx[dd]; }
  }
}

void init_area()
{
  int ii=0, jj=0, kk=0, loc, dd;
  for (ii=istart[0]; ii<=istop[0]; ii++) {
#if (NDIM>1)
    for (jj=istart[1]; jj<=istop[1]; jj++) {
#endif
#if (NDIM==3)
      for (kk=istart[2]; kk<=istop[2]; kk++) {
#endif
        for (loc=0; loc<NDIM; loc++) {
          ND_ELEM_LINEAR(geom,ii,jj,kk).area[loc] = 1.0;
          DLOOP { ND_ELEM_LINEAR(geom,ii,jj,kk).area[loc] *= dx[dd]; }
          ND_ELEM_LINEAR(geom,ii,jj,kk).area[loc] /= dx[loc];
        }
#if (NDIM==3)
      }
#endif
#if (NDIM>1)
    }
#endif
  }
}

void init_conn()
{
  int ii=0, jj=0, kk=0;
  ZLOOP { memset(&ND_ELEM_LINEAR(geom,ii,jj,kk).conn[0][0][0], 0, 27*sizeof(double)); }
}

void init_gcov()
{
  int ii=0, jj=0, kk=0, loc, i;
  ZGLOOP {
    for (loc=0; loc<=NDIM; loc++)
      for (i=0; i<SPACEDIM; i++) ND_ELEM_LINEAR(geom,ii,jj,kk).gcov[loc][i] = 1.0;
  }
}

void init_gcon()
{
  int ii=0, jj=0, kk=0, i;
  ZGLOOP {
    for (i=0; i<SPACEDIM; i++) ND_ELEM_LINEAR(geom,ii,jj,kk).gcon[i] = 1.0;
  }
}

void init_scale()
{
  int ii=0, jj=0, kk=0, loc, dd;
  ZGLOOP {
    for (loc=0; loc<=NDIM; loc++) SLOOP { ND_ELEM_LINEAR(geom,ii,jj,kk).scale[loc][dd] = 1.0; }
  }
}

double r_of_x(r_of_x_struct_t rx, double x) { (void)rx; return x; }
double th_of_x(th_of_x_struct_t thx, double x) { (void)thx; return x; }
double dr_dx(double x) { (void)x; return 1.0; }
double dth_dx(double x) { (void)x; return 1.0; }
double x_of_r(double r) { return r; }
double rtrans_solve(double dxx, double rout) { (void)dxx; (void)rout; return 1.0; }
