/*
 * Device/DeviceInterface.h in place of the reference's
 * (V_02_2015/src/Device/DeviceInterface.h:16-95): the reference's KDevice
 * wrapper (Interface/KDevice.h) compiles against this header unchanged and
 * links against libblaze_b200.so.
 *
 * KDevice.h includes "../Device/DeviceInterface.h" relative to itself; to
 * have it take this file, put include/kdevice/Device and include/ ahead of
 * the reference's directories and stop the compiler from looking beside the
 * including file first (g++ -I include/kdevice/Device -I include -I- ...).
 */
#ifndef BLAZE_KDEVICE_DEVICEINTERFACE_H_
#define BLAZE_KDEVICE_DEVICEINTERFACE_H_

#include "blaze_dem.h"  /* the live functions: extern "C", int status */

/* Declared by the reference but never defined (DeviceInterface.h:57, 65, 78,
 * 92-94); KDevice.h names them in inline members a headless driver does not
 * call, so no definition is needed. */
void End_Packing(SimulationInfo* SimInfo, WOBJ* WorldOBJ);
void Device_World_Interaction(void);
void Device_World_InteractionS(void);
void Device_Body_Body_Interaction(void);

#endif
