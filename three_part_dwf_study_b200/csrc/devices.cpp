// Device selection for processes that run side by side on one host: the
// study driver runs its four cases concurrently (scripts/run_three_part_study.py
// :166-169), each as separate generate/analyze processes; handing each new
// process the next GPU in turn spreads them over the host's GPUs.
#include <fcntl.h>
#include <sys/file.h>
#include <unistd.h>

#include <cstdio>
#include <cstdlib>
#include <cstring>

#include <cuda_runtime.h>

#include "../../include/dwf_b200.h"

extern "C" {

int dwf_device_count(int* count)
{
    if (!count)
        return DWF_BAD_ARG;
    *count = 0;
    int n = 0;
    if (cudaGetDeviceCount(&n) != cudaSuccess)
    {
        cudaGetLastError();  // no device here: leave no error pending for later calls
        return DWF_CUDA_ERROR;
    }
    *count = n;
    return DWF_OK;
}

int dwf_round_robin_device(int ndevices, const char* counter_path, int* device)
{
    if (ndevices < 1 || !counter_path || !*counter_path || !device)
        return DWF_BAD_ARG;
    const int fd = open(counter_path, O_RDWR | O_CREAT, 0666);
    if (fd < 0)
        return DWF_BAD_ARG;
    int st = DWF_OK;
    if (flock(fd, LOCK_EX) != 0)
    {
        close(fd);
        return DWF_BAD_ARG;
    }
    char buf[32] = {0};
    const ssize_t got = pread(fd, buf, sizeof(buf) - 1, 0);
    long next = got > 0 ? std::strtol(buf, nullptr, 10) : 0;
    if (next < 0)
        next = 0;
    *device = int(next % ndevices);
    const int len = std::snprintf(buf, sizeof(buf), "%ld\n", next + 1);
    if (ftruncate(fd, 0) != 0 || pwrite(fd, buf, size_t(len), 0) != len)
        st = DWF_BAD_ARG;
    flock(fd, LOCK_UN);
    close(fd);
    return st;
}

}  // extern "C"
