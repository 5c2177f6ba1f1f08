/* The C ABI header compiles as C99 and every declared entry point links. */
#include <stdio.h>

#include "svg_b200.h"

int main(void) {
    svg_build_opts o;
    svg_build_opts_default(&o);
    printf("%s K=%d\n", svg_version(), o.K);
    /* take the address of every entry point so the link resolves each one */
    void* fns[] = {
        (void*)svg_last_error, (void*)svg_version, (void*)svg_mesh_load_obj, (void*)svg_mesh_from_arrays,
        (void*)svg_mesh_upload, (void*)svg_mesh_free, (void*)svg_mesh_counts, (void*)svg_mesh_export,
        (void*)svg_build_opts_default, (void*)svg_build, (void*)svg_build_autotune, (void*)svg_graph_stats, (void*)svg_graph_source_stats,
        (void*)svg_graph_free, (void*)svg_graph_set_query_form, (void*)svg_graph_counts, (void*)svg_graph_copy_csr,
        (void*)svg_graph_copy_nodes, (void*)svg_graph_device_csr, (void*)svg_graph_save, (void*)svg_graph_load,
        (void*)svg_sssd_batch, (void*)svg_msad_batch, (void*)svg_msad_batch_paths, (void*)svg_sssd_path,
        (void*)svg_sssd_batch_device, (void*)svg_msad_batch_device, (void*)svg_build_rows_static,
        (void*)svg_server_opts_default, (void*)svg_server_create, (void*)svg_server_free,
        (void*)svg_server_add_graph, (void*)svg_server_submit_build, (void*)svg_server_submit_sssd,
        (void*)svg_server_submit_msad, (void*)svg_server_submit_msad_into, (void*)svg_server_wait,
        (void*)svg_server_poll, (void*)svg_server_take, (void*)svg_server_stats, (void*)svg_server_resident,
        (void*)svg_trim_device_cache, (void*)svg_device_memory, (void*)svg_timer_mark, (void*)svg_device_fp64_rate,
    };
    int n = 0;
    for (size_t i = 0; i < sizeof(fns) / sizeof(fns[0]); ++i) n += fns[i] != 0;
    printf("%d entry points\n", n);
    return 0;
}
