/* A C caller of the drop-in path with no Python in the loop: reads a plan in
 * the reference's INI format and a physics file, transports every field's
 * histories on GPU 0 and writes the dose file the way the reference's
 * write_dose does (output.c:873-918).
 *
 *   plan_dose <plan.ini> <physics file> [max histories per field]
 *
 * Prints the dose file's name. Built and run by tests/test_c_boundary.py. */
#include <stdio.h>
#include <stdlib.h>
#include "gegs.h"
#include "gegs_plan.h"

int main(int argc, char **argv)
{
    if (argc < 3) {
        fprintf(stderr, "usage: %s plan.ini physics_file [max_histories_per_field]\n", argv[0]);
        return 2;
    }
    char msg[512];
    gegs_plan *plan = NULL;
    uint64_t cap = argc > 3 ? strtoull(argv[3], NULL, 10) : 0;
    if (gegs_plan_load(argv[1], argv[2], cap, &plan, msg, sizeof msg) != GEGS_OK) {
        fprintf(stderr, "plan: %s\n", msg);
        return 1;
    }
    gegs_engine *e = NULL;
    if (gegs_create(0, &e) != GEGS_OK || gegs_set_physics(e, gegs_plan_physics(plan)) != GEGS_OK ||
        gegs_set_scene(e, gegs_plan_scene(plan)) != GEGS_OK ||
        gegs_run(e, 0, gegs_plan_histories(plan), NULL) != GEGS_OK) {
        fprintf(stderr, "transport: %s\n", gegs_last_error(e));
        return 1;
    }
    const uint64_t nvox = gegs_plan_nvox(plan);
    int64_t *tally = (int64_t *)malloc(nvox * sizeof(int64_t));
    float *dose = (float *)malloc(nvox * sizeof(float));
    char path[1024];
    if (gegs_get_tally(e, tally, nvox) != GEGS_OK || gegs_plan_dose(plan, tally, dose, nvox) != GEGS_OK ||
        gegs_plan_write_dose(plan, dose, nvox, path, sizeof path) != GEGS_OK) {
        fprintf(stderr, "dose: %s\n", gegs_last_error(e));
        return 1;
    }
    printf("%s\n", path);
    free(tally);
    free(dose);
    gegs_destroy(e);
    gegs_plan_free(plan);
    return 0;
}
