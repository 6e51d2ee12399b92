/* A time() that always answers the same instant, preloaded (LD_PRELOAD) into
 * the CLI's play and train commands so that their srand(time(NULL)) seeds the
 * same spawn sequence on every run: the reference CLI and the same CLI linked
 * to this library then play the same game and their transcripts compare. */
#include <time.h>

time_t time(time_t *t)
{
    const time_t now = 1733300000;
    if (t) *t = now;
    return now;
}
