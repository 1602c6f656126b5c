/* Stand-in for the difxmessage UDP status library: alert levels and the one
 * send call that the reference's Alert streams make, plus what Visibility
 * and core.h name (the status send, its state value, the STA record type,
 * left incomplete). The oracle build routes alerts to stderr (level <= ERROR)
 * or drops them, and drops status messages. */
#ifndef ORACLE_REFSTUB_DIFXMESSAGE_H
#define ORACLE_REFSTUB_DIFXMESSAGE_H
#define DIFX_ALERT_LEVEL_FATAL 0
#define DIFX_ALERT_LEVEL_SEVERE 1
#define DIFX_ALERT_LEVEL_ERROR 2
#define DIFX_ALERT_LEVEL_WARNING 3
#define DIFX_ALERT_LEVEL_INFO 4
#define DIFX_ALERT_LEVEL_VERBOSE 5
#define DIFX_ALERT_LEVEL_DEBUG 6
#define DIFX_ALERT_LEVEL_DO_NOT_SEND 7
#define DIFX_MESSAGE_PARAM_LENGTH 32
#define DIFX_STATE_RUNNING 4
typedef struct DifxMessageSTARecord DifxMessageSTARecord;
#ifdef __cplusplus
extern "C" {
#endif
int difxMessageSendDifxAlert(const char *alertMessage, int severity);
int difxMessageSendDifxStatus3(int state, const char *message, double visMJD, int numdatastreams, float *weight,
                               double mjdStart, double mjdStop);
int difxMessageSendDifxDiagnosticBufferStatus(int threadid, int numelements, int startelement, int numactiveelements);
int difxMessageSendDifxDiagnosticDataConsumed(long long bytes);
int difxMessageSendDifxDiagnosticInputDatarate(double bytespersec);
#ifdef __cplusplus
}
#endif
#endif
