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
    F(rl_stats, max_level);
    return 0;
}
