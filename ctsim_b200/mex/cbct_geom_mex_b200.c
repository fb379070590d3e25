/*
 * MATLAB MEX gateway onto the B200 projector library -- a drop-in for the
 * reference's cbct_geom_mex / cbct_dd_cuda / cbct_sf_cuda / cbct_back_pd_cuda.
 *
 *   sino = cbct_geom_mex_b200('proj,dd', int32(nxyz), single(dxyz), single(cxyz),
 *              int32(nuv), single(duv), single(cuv), single(SAD), single(ADD),
 *              single(SDD), int32(noViews), double(betas), single(couchZ),
 *              int32(flatPanel), single(img), logical(map));
 *   img  = cbct_geom_mex_b200('back,tf', ..., single(sino), logical(map));
 *
 * Same 16 arguments, types, checks and error messages as the reference gateway
 * (geom/cbct/cbct_geom_mex.c:23-326); the projection itself is one call to
 * ctsim_cbct_geom (include/ctsim_b200.h).  Build (MATLAB, Linux):
 *
 *   mex -I<repo>/include cbct_geom_mex_b200.c -L<repo>/ctsim_b200/_lib -lctsim_b200
 *
 * and call it from geom/shell/forwardProjectMex.m / backProjectMex.m in place of
 * cbct_geom_mex.  Called with no arguments and no outputs it prints its usage, as the
 * reference gateway prints its help (geom/cbct/cbct_geom_mex.c:317-320).
 */
#include <string.h>

#include "mex.h"
#include "ctsim_b200.h"

static const char *ARG_TYPES[] = {"proj,dd", "proj,tf", "back,dd", "back,tf", "back,pd", "back,hpd", "back,var"};

static int known_type(const char *t)
{
    for (size_t i = 0; i < sizeof(ARG_TYPES) / sizeof(ARG_TYPES[0]); i++)
        if (!strcmp(t, ARG_TYPES[i])) return 1;
    return 0;
}

static void usage(void)
{
    mexPrintf("\n"
              "  sino = cbct_geom_mex_b200(type, int32([nx ny nz]), single([dx dy dz]), single([ox oy oz]),\n"
              "             int32([nu nv]), single([du dv]), single([ou ov]), single(SAD), single(ADD),\n"
              "             single(SDD), int32(noViews), double(betas), single(couchZ),\n"
              "             int32(flatPanel), single(data), logical(map))\n"
              "  type: proj,dd | proj,tf  (data: image [nx ny nz] -> sinogram [nv nu noViews])\n"
              "        back,dd | back,tf | back,pd | back,hpd | back,var  (sinogram -> image)\n");
}

void mexFunction(int nlhs, mxArray *plhs[], int nrhs, const mxArray *prhs[])
{
    char type[16];
    if (!nlhs && !nrhs) {
        usage();
        return;
    }
    if (nrhs != 16 || !mxIsChar(prhs[0]) || mxGetString(prhs[0], type, sizeof(type)))
        mexErrMsgTxt("The 1st argument is invalid! \n");
    if (!known_type(type)) mexErrMsgTxt("Error: unknown geom type. \n");

    const int *nxyz = (const int *)mxGetData(prhs[1]);
    const float *dxyz = (const float *)mxGetData(prhs[2]);
    const float *cxyz = (const float *)mxGetData(prhs[3]);
    const int *nuv = (const int *)mxGetData(prhs[4]);
    const float *duv = (const float *)mxGetData(prhs[5]);
    const float *cuv = (const float *)mxGetData(prhs[6]);
    const float sad = *(const float *)mxGetData(prhs[7]);
    const float add = *(const float *)mxGetData(prhs[8]);
    const float sdd = *(const float *)mxGetData(prhs[9]);
    const int noviews = *(const int *)mxGetData(prhs[10]);
    const int detector_type = *(const int *)mxGetData(prhs[13]);
    const int nx = nxyz[0], ny = nxyz[1], nz = nxyz[2], nu = nuv[0], nv = nuv[1];
    const mxArray *mx_betas = prhs[11], *mx_couchz = prhs[12], *mx_data = prhs[14], *mx_map = prhs[15];

    /* checks of geom/cbct/cbct_geom_mex.c:78-107 and :190-221 */
    if ((size_t)noviews != mxGetM(mx_betas) * mxGetN(mx_betas) || !mxIsDouble(mx_betas) || mxIsComplex(mx_betas))
        mexErrMsgTxt("Error: mx_betas must have noviews X 1 double array.\n");
    if ((size_t)noviews != mxGetM(mx_couchz) * mxGetN(mx_couchz) || !mxIsSingle(mx_couchz))
        mexErrMsgTxt("Error: mx_couchz must have noviews X 1 double array.\n");
    const mwSize *dm = mxGetDimensions(mx_map);
    if (mxGetNumberOfDimensions(mx_map) < 2 || (mwSize)nx != dm[0] || (mwSize)ny != dm[1] || !mxIsLogical(mx_map))
        mexErrMsgTxt("Error: mx_map must have [nx ny] bool array.\n");
    const mwSize *dd = mxGetDimensions(mx_data);
    const mwSize nd = mxGetNumberOfDimensions(mx_data);
    mwSize dims[3];
    if (!strncmp(type, "proj", 4)) {
        if (nd < 2 || dd[0] != (mwSize)nx || dd[1] != (mwSize)ny || (nd > 2 ? dd[2] : 1) != (mwSize)nz ||
            !mxIsSingle(mx_data))
            mexErrMsgTxt("Error: mx_image must have [nx ny nz] float array.\n");
        dims[0] = nv; dims[1] = nu; dims[2] = noviews;
    } else {
        if (nd < 2 || dd[0] != (mwSize)nv || dd[1] != (mwSize)nu || (nd > 2 ? dd[2] : 1) != (mwSize)noviews ||
            !mxIsSingle(mx_data))
            mexErrMsgTxt("Error: mx_proj must have [nv nu noviews] float array.\n");
        dims[0] = nx; dims[1] = ny; dims[2] = nz;
    }
    plhs[0] = mxCreateNumericArray(3, dims, mxSINGLE_CLASS, mxREAL);
    (void)nlhs;
    if (!ctsim_cbct_geom(type, nx, ny, nz, dxyz[0], dxyz[1], dxyz[2], cxyz[0], cxyz[1], cxyz[2], nu, nv, duv[0],
                         duv[1], cuv[0], cuv[1], sad, add, sdd, noviews, (const double *)mxGetData(mx_betas),
                         (const float *)mxGetData(mx_couchz), detector_type, (const float *)mxGetData(mx_data),
                         (float *)mxGetData(plhs[0]), (const bool *)mxGetData(mx_map))) {
        mexPrintf("%s\n", ctsim_last_error());
        mexErrMsgTxt("Error: cbct_geom_mex() failed. \n");
    }
}
