/* Minimal stand-in for <SDL3/SDL.h> so the reference's CPU loader / cull / sort
 * translation units compile without SDL3.  Test infrastructure only: it is used
 * to build oracle/_ref, never linked into the product library. */
#pragma once
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#define SDL_malloc malloc
#define SDL_free free
#define SDL_strcmp strcmp
#define SDL_Log(...) (fprintf(stderr, __VA_ARGS__), fputc('\n', stderr))
/* The reference's LOG(flags, fmt, ...) logging macro, silenced. */
#ifndef LOG
#define LOG(flags, ...) ((void)0)
#endif
