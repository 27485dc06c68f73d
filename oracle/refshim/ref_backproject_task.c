/* Drives the reference's own `backproject` task (src/ufo-backproject-task.c,
 * compiled in this translation unit against the CPU shims): properties, setup,
 * get_requisition (sin/cos LUTs) and process (backproject.cl on the CPU).
 * Test infrastructure only. */
#include "ufo-backproject-task.c"
#include "refshim_internal.h"
#include <stdio.h>

int ref_backproject_run(float *sino, unsigned width, unsigned height, float *out, size_t out_capacity,
                        unsigned num_projections, unsigned offset, double axis_pos, double angle_step,
                        double angle_offset, int mode, unsigned roi_x, unsigned roi_y, unsigned roi_width,
                        unsigned roi_height, unsigned *out_w, unsigned *out_h, char *err, int errlen)
{
    UfoBackprojectTaskPrivate priv;
    UfoBackprojectTask task;
    GError *e = NULL;
    GValue v;
    UfoBuffer in, outb;
    UfoBuffer *inputs[1];
    UfoRequisition req;

    memset(&priv, 0, sizeof priv);
    memset(&task, 0, sizeof task);
    task.priv = &priv;
    ufo_backproject_task_init(&task);
    v.data.u = num_projections;
    ufo_backproject_task_set_property((GObject *)&task, PROP_NUM_PROJECTIONS, &v, NULL);
    v.data.u = offset;
    ufo_backproject_task_set_property((GObject *)&task, PROP_OFFSET, &v, NULL);
    v.data.d = axis_pos;
    ufo_backproject_task_set_property((GObject *)&task, PROP_AXIS_POSITION, &v, NULL);
    v.data.d = angle_step;
    ufo_backproject_task_set_property((GObject *)&task, PROP_ANGLE_STEP, &v, NULL);
    v.data.d = angle_offset;
    ufo_backproject_task_set_property((GObject *)&task, PROP_ANGLE_OFFSET, &v, NULL);
    v.data.i = mode;
    ufo_backproject_task_set_property((GObject *)&task, PROP_MODE, &v, NULL);
    v.data.u = roi_x;
    ufo_backproject_task_set_property((GObject *)&task, PROP_ROI_X, &v, NULL);
    v.data.u = roi_y;
    ufo_backproject_task_set_property((GObject *)&task, PROP_ROI_Y, &v, NULL);
    v.data.u = roi_width;
    ufo_backproject_task_set_property((GObject *)&task, PROP_ROI_WIDTH, &v, NULL);
    v.data.u = roi_height;
    ufo_backproject_task_set_property((GObject *)&task, PROP_ROI_HEIGHT, &v, NULL);

    ufo_backproject_task_setup((UfoTask *)&task, NULL, &e);
    refshim_buffer_init(&in, sino, 2, width, height, 1);
    inputs[0] = &in;
    ufo_backproject_task_get_requisition((UfoTask *)&task, inputs, &req, &e);
    if (e) {
        snprintf(err, errlen, "%s", e->message);
        free(e);
        return -1;
    }
    *out_w = (unsigned)req.dims[0];
    *out_h = (unsigned)req.dims[1];
    if ((size_t)req.dims[0] * req.dims[1] > out_capacity) {
        snprintf(err, errlen, "output buffer too small");
        return -2;
    }
    refshim_buffer_init(&outb, out, 2, req.dims[0], req.dims[1], 1);
    ufo_backproject_task_process((UfoTask *)&task, inputs, &outb, &req);
    return 0;
}
