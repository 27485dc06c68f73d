/* Drives the reference's own `filter` task (src/ufo-filter-task.c, compiled in
 * this translation unit against the CPU shims) through its property setters,
 * setup, get_requisition and process.  Test infrastructure only. */
#include "ufo-filter-task.c"
#include "refshim_internal.h"
#include <stdio.h>

int ref_filter_run(int filter, float cutoff, float order, float tau, float theta, float scale, unsigned width2,
                   unsigned rows, float *spectrum_in, float *spectrum_out, float *coeff_out, char *err, int errlen)
{
    UfoFilterTaskPrivate priv;
    UfoFilterTask task;
    GError *e = NULL;
    GValue v;
    UfoBuffer in, out;
    UfoBuffer *inputs[1];
    UfoRequisition req;

    memset(&priv, 0, sizeof priv);
    memset(&task, 0, sizeof task);
    task.priv = &priv;
    ufo_filter_task_init(&task);
    v.data.i = filter;
    ufo_filter_task_set_property((GObject *)&task, PROP_FILTER, &v, NULL);
    v.data.f = cutoff;
    ufo_filter_task_set_property((GObject *)&task, PROP_CUTOFF, &v, NULL);
    v.data.f = order;
    ufo_filter_task_set_property((GObject *)&task, PROP_BW_ORDER, &v, NULL);
    v.data.f = tau;
    ufo_filter_task_set_property((GObject *)&task, PROP_FB_TAU, &v, NULL);
    v.data.f = theta;
    ufo_filter_task_set_property((GObject *)&task, PROP_FB_THETA, &v, NULL);
    v.data.f = scale;
    ufo_filter_task_set_property((GObject *)&task, PROP_SCALE, &v, NULL);
    ufo_filter_task_setup((UfoTask *)&task, NULL, &e);
    refshim_buffer_init(&in, spectrum_in, 2, width2, rows ? rows : 1, 1);
    refshim_buffer_init(&out, spectrum_out, 2, width2, rows ? rows : 1, 1);
    inputs[0] = &in;
    ufo_filter_task_get_requisition((UfoTask *)&task, inputs, &req, &e);
    if (e) {
        snprintf(err, errlen, "%s", e->message);
        free(e);
        return -1;
    }
    if (spectrum_in && spectrum_out)
        ufo_filter_task_process((UfoTask *)&task, inputs, &out, &req);
    if (coeff_out)
        memcpy(coeff_out, priv.filter_mem->host, width2 * sizeof(float));
    return 0;
}
