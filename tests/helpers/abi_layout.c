/* Prints the sizes and field offsets of the C-ABI structs. */
#include <stddef.h>
#include <stdio.h>

#include "../../include/relearn_b200.h"

#define F(T, f) printf("%s.%s %zu\n", #T, #f, offsetof(T, f))

int main(void) {
    printf("rl_config %zu\n", sizeof(rl_config));
    printf("rl_request %zu\n", sizeof(rl_request));
    printf("rl_synapse %zu\n", sizeof(rl_synapse));
    printf("rl_stats %zu\n", sizeof(rl_stats));
    F(rl_config, seed);
    F(rl_config, box_min);
    F(rl_config, theta);
    F(rl_config, growth_rate);
    F(rl_config, conductance);
    F(rl_config, device);
    F(rl_config, precision);
    F(rl_config, kernel_type);
    F(rl_config, kernel_k);
    F(rl_config, kernel_scale);
    F(rl_config, linear_cutoff);
    F(rl_stats, max_level);
    F(rl_stats, nodes_touched);
    printf("rl_network %zu\n", sizeof(rl_network));
    printf("rl_tuning %zu\n", sizeof(rl_tuning));
    printf("RL_NUM_SEARCH_SHAPES %d\n", RL_NUM_SEARCH_SHAPES);
    printf("RL_NUM_ACT_SHAPES %d\n", RL_NUM_ACT_SHAPES);
    printf("rl_serve_config %zu\n", sizeof(rl_serve_config));
    printf("rl_serve_request %zu\n", sizeof(rl_serve_request));
    printf("rl_serve_done %zu\n", sizeof(rl_serve_done));
    F(rl_network, growth_rate);
    F(rl_serve_config, slots);
    F(rl_serve_config, use_graphs);
    F(rl_serve_request, xyz);
    F(rl_serve_request, grown);
    F(rl_serve_request, steps);
    F(rl_serve_request, keep_state);
    F(rl_serve_done, t_submit);
    F(rl_serve_done, num_synapses);
    F(rl_serve_done, neuron_steps);
    return 0;
}
