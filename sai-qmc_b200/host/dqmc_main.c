/* dqmc_gpu: command-line driver, a drop-in for the reference program
 * (`dqmc input.txt`, SAI-QMC src/main.c:603) running on one GPU. */
#include <stdio.h>

#include "dqmc_host.h"

int main(int argc, char **argv)
{
    if (argc < 2) {
        fprintf(stderr, "usage: %s input.txt\n", argv[0]);
        return 1;
    }
    return dqmc_host_run(argv[1]);
}
