/*
 * MATLAB MEX gateway onto the B200 fan-beam projectors -- a drop-in for the
 * reference's 2-D fbct_geom_mex.
 *
 *   sino = fbct_geom_mex_b200('proj,dd', int32(nxy), single(dxy), single(cxy),
 *              int32(nu), single(du), single(cu), single(SAD), single(ADD),
 *              single(SDD), int32(noViews), double(betas), int32(flatPanel), single(img));
 *   img  = fbct_geom_mex_b200('back,tf', ..., single(sino));
 *
 * Same 14 arguments, types, checks and error messages as the reference gateway
 * (geom/fbct/fbct_geom_mex.c:43-278) for "proj,dd", "proj,tf", "back,dd" and
 * "back,tf"; the projection itself is one call to ctsim_fbct_geom
 * (include/ctsim_b200.h).  Image [nx ny], sinogram [nu noViews].  Build (MATLAB, Linux):
 *
 *   mex -I<repo>/include fbct_geom_mex_b200.c -L<repo>/ctsim_b200/_lib -lctsim_b200
 */
#include <string.h>

#include "mex.h"
#include "ctsim_b200.h"

static const char *ARG_TYPES[] = {"proj,dd", "proj,tf", "back,dd", "back,tf"};

static int known_type(const char *t)
{
    for (size_t i = 0; i < sizeof(ARG_TYPES) / sizeof(ARG_TYPES[0]); i++)
        if (!strcmp(t, ARG_TYPES[i])) return 1;
    return 0;
}

static void usage(void)
{
    mexPrintf("\n"
              "  sino = fbct_geom_mex_b200(type, int32([nx ny]), single([dx dy]), single([ox oy]),\n"
              "             int32(nu), single(du), single(ou), single(SAD), single(ADD), single(SDD),\n"
              "             int32(noViews), double(betas), int32(flatPanel), single(data))\n"
              "  type: proj,dd | proj,tf  (image [nx ny] -> sinogram [nu noViews])\n"
              "        back,dd | back,tf  (sinogram -> image)\n");
}

void mexFunction(int nlhs, mxArray *plhs[], int nrhs, const mxArray *prhs[])
{
    char type[16];
    if (!nlhs && !nrhs) {  /* usage, as with the cone-beam gateway */
        usage();
        return;
    }
    if (nrhs < 1 || !mxIsChar(prhs[0]) || mxGetString(prhs[0], type, sizeof(type)))
        mexErrMsgTxt("The 1st argument is invalid! \n");
    if (nrhs != 14 || nlhs != 1) mexErrMsgTxt("Error: incorrect number of arguments. \n");
    if (!known_type(type)) mexErrMsgTxt("Error: unknown geom type. \n");

    const int *nxy = (const int *)mxGetData(prhs[1]);
    const float *dxy = (const float *)mxGetData(prhs[2]);
    const float *cxy = (const float *)mxGetData(prhs[3]);
    const int nu = *(const int *)mxGetData(prhs[4]);
    const float du = *(const float *)mxGetData(prhs[5]);
    const float cu = *(const float *)mxGetData(prhs[6]);
    const float sad = *(const float *)mxGetData(prhs[7]);
    const float add = *(const float *)mxGetData(prhs[8]);
    const float sdd = *(const float *)mxGetData(prhs[9]);
    const int noviews = *(const int *)mxGetData(prhs[10]);
    const int detector_type = *(const int *)mxGetData(prhs[12]);
    const int nx = nxy[0], ny = nxy[1];
    const mxArray *mx_betas = prhs[11], *mx_data = prhs[13];

    /* checks of geom/fbct/fbct_geom_mex.c:91-104 and :177-190 */
    if ((size_t)noviews != mxGetM(mx_betas) * mxGetN(mx_betas) || !mxIsDouble(mx_betas) || mxIsComplex(mx_betas))
        mexErrMsgTxt("Error: mx_betas must have noviews X 1 double array.\n");
    const mwSize *dd = mxGetDimensions(mx_data);
    mwSize dims[2];
    if (!strncmp(type, "proj", 4)) {
        if (mxGetNumberOfDimensions(mx_data) < 2 || dd[0] != (mwSize)nx || dd[1] != (mwSize)ny || !mxIsSingle(mx_data))
            mexErrMsgTxt("Error: mx_image must have [nx ny] float array.\n");
        dims[0] = nu; dims[1] = noviews;
    } else {
        if (mxGetNumberOfDimensions(mx_data) < 2 || dd[0] != (mwSize)nu || dd[1] != (mwSize)noviews ||
            !mxIsSingle(mx_data))
            mexErrMsgTxt("Error: mx_proj must have [nu noviews] float array.\n");
        dims[0] = nx; dims[1] = ny;
    }
    plhs[0] = mxCreateNumericArray(2, dims, mxSINGLE_CLASS, mxREAL);
    if (!ctsim_fbct_geom(type, nx, ny, dxy[0], dxy[1], cxy[0], cxy[1], nu, du, cu, sad, add, sdd, noviews,
                         (const double *)mxGetData(mx_betas), detector_type, (const float *)mxGetData(mx_data),
                         (float *)mxGetData(plhs[0]))) {
        mexPrintf("%s\n", ctsim_last_error());
        mexErrMsgTxt("Error: fbct_geom_mex() failed. \n");
    }
}
