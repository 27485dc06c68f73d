/* Drives the reference's own `stacked-backproject` task
 * (src/ufo-stacked-backproject-task.c, compiled in this translation unit
 * against the CPU shims): properties through the task's set_property, setup,
 * get_requisition and process on one sinogram stack [z][projections][width].
 * Its kernels (src/kernels/stacked-backproject.cl: interleave into an image
 * array, 16x16 work-groups that reduce partial sums in local memory between
 * barriers, uninterleave) are compiled for the CPU by ref_clc_jit.cpp, which
 * runs each work-group as one OpenMP team.  Test infrastructure only. */
#include "ufo-stacked-backproject-task.c"
#include "refshim_internal.h"

typedef struct {
    UfoStackedBackprojectTask task;
    UfoStackedBackprojectTaskPrivate *priv;
} RefStacked;

void *ref_stacked_new(void)
{
    RefStacked *g = (RefStacked *)calloc(1, sizeof(RefStacked));
    g->priv = (UfoStackedBackprojectTaskPrivate *)calloc(1, sizeof(UfoStackedBackprojectTaskPrivate));
    g->task.priv = g->priv;
    ufo_stacked_backproject_task_init(&g->task);
    return g;
}

/* Set one property by its reference name (precision-mode by value nick).
 * Returns 0, or -1 for an unknown name or nick. */
int ref_stacked_set(void *handle, const char *name, double value, const char *nick)
{
    RefStacked *g = (RefStacked *)handle;
    static const struct {
        const char *name;
        guint id;
        GType type;
    } props[] = {
        {"num-projections", PROP_NUM_PROJECTIONS, G_TYPE_UINT}, {"offset", PROP_OFFSET, G_TYPE_UINT},
        {"axis-pos", PROP_AXIS_POSITION, G_TYPE_DOUBLE},        {"angle-step", PROP_ANGLE_STEP, G_TYPE_DOUBLE},
        {"angle-offset", PROP_ANGLE_OFFSET, G_TYPE_DOUBLE},     {"roi-x", PROP_ROI_X, G_TYPE_UINT},
        {"roi-y", PROP_ROI_Y, G_TYPE_UINT},                     {"roi-width", PROP_ROI_WIDTH, G_TYPE_UINT},
        {"roi-height", PROP_ROI_HEIGHT, G_TYPE_UINT},           {"precision-mode", PROP_PRECISION, G_TYPE_ENUM},
    };
    GValue v = G_VALUE_INIT;
    unsigned k;
    for (k = 0; k < sizeof props / sizeof props[0]; k++)
        if (!strcmp(props[k].name, name)) break;
    if (k == sizeof props / sizeof props[0]) return -1;
    g_value_init(&v, props[k].type);
    if (props[k].type == G_TYPE_ENUM) {
        const GEnumValue *t;
        for (t = precision_values; t->value_nick; t++)
            if (nick && !strcmp(t->value_nick, nick)) break;
        if (!t->value_nick) return -1;
        g_value_set_enum(&v, t->value);
    } else if (props[k].type == G_TYPE_UINT) {
        g_value_set_uint(&v, (guint)value);
    } else {
        g_value_set_double(&v, value);
    }
    ufo_stacked_backproject_task_set_property((GObject *)&g->task, props[k].id, &v, NULL);
    return 0;
}

/* Run the task on `slices` sinograms of `rows` x `width` floats.  dims gets the
 * requisition (x, y, z); `out` (zeroed by the caller) receives the volume when
 * it holds dims[0] * dims[1] * dims[2] floats.  Returns 0, or -1 with the
 * task's GError message in err. */
int ref_stacked_run(void *handle, float *sino, unsigned width, unsigned rows, unsigned slices, float *out,
                    size_t out_floats, unsigned *dims, char *err, int errlen)
{
    RefStacked *g = (RefStacked *)handle;
    UfoTask *task = (UfoTask *)&g->task;
    GError *e = NULL;
    UfoBuffer in, ob;
    UfoBuffer *inputs[1] = {&in};
    UfoRequisition req;

    memset(&req, 0, sizeof req);
    ufo_stacked_backproject_task_setup(task, NULL, &e);
    if (!e) {
        refshim_buffer_init(&in, sino, 3, width, rows, slices);
        ufo_stacked_backproject_task_get_requisition(task, inputs, &req, &e);
    }
    if (e) {
        snprintf(err, errlen, "%s", e->message);
        free(e);
        return -1;
    }
    dims[0] = (unsigned)req.dims[0];
    dims[1] = (unsigned)req.dims[1];
    dims[2] = (unsigned)req.dims[2];
    if (!out || (size_t)dims[0] * dims[1] * dims[2] > out_floats) return 0;
    refshim_buffer_init(&ob, out, 3, dims[0], dims[1], dims[2]);
    ufo_stacked_backproject_task_process(task, inputs, &ob, &req);
    return 0;
}
