/*
 * Stand-in for the reference's Util/Logger.h: the kernel files log nothing,
 * so only the macro names exist here (see Common/Common.h of this directory).
 */
#ifndef PFD_REF_STUB_LOGGER_H
#define PFD_REF_STUB_LOGGER_H

#define LOG_DEBUG(...) ((void)0)
#define LOG_INFO(...) ((void)0)
#define LOG_WARN(...) ((void)0)
#define LOG_ERROR(...) ((void)0)

#endif
