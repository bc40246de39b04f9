// The timer macros the reference's sources and drivers use
// (utils/chtimer/CH_Timer.H:340-372).  On the GPU, kernels run asynchronously
// and are timed with CUDA events and ncu instead, so these compile to nothing,
// exactly as the reference's own CH_NTIMER build does.
#ifndef SNS_CH_TIMER_H
#define SNS_CH_TIMER_H

#define CH_TIMER(name, tpointer) (void)0
#define CH_TIME(name) (void)0
#define CH_TIMELEAF(name) (void)0
#define CH_TIMERS(name) (void)0
#define CH_START(tpointer) (void)0
#define CH_STOP(tpointer) (void)0
#define CH_STOPV(tpointer, val) (void)0
#define CH_TIMER_REPORT() (void)0
#define CH_TIMER_RESET() (void)0
#define CH_TIMER_PRUNE(threshold) (void)0

#endif
